"""Domain-decomposed RK4 over several GPUs, one process per GPU.

Replaces the reference's MPI rank loop: MemoryNetwork::communicate_face_solution
(src/memory/memory_network.cpp:55-175) becomes a per-stage exchange of boundary
coefficient slices over a torch.distributed process group (NCCL over NVLink on
GPUs, gloo in the CPU tests), overlapped with the stage kernel on the interior
elements:

    pack(stage input) -> isend/irecv per peer -> stage(interior elements)
    -> wait -> unpack into the ghosts -> stage(boundary elements)

all ordered on the context's CUDA stream (the transport's stream waits for the
pack, the context's stream waits for the transport before the unpack).  Every
rank takes the same collective steps in the same order.

Two transports: "device" exchanges the device buffers through the process
group's backend (NCCL between GPUs); "host" stages them through pinned host
buffers and exchanges those over a CPU backend (gloo) -- the same stage order
with the host in the middle, which also lets several ranks share one GPU
(each rank's kernels run on its own stream and no kernel waits on another
rank: the host orders pack -> copy out -> exchange -> copy in -> unpack).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

import dg_b200


class HaloExchange:
    """Send / receive buffers of one rank's halo and their exchange.

    ``peers`` is [(peer rank, slice offset, slice count)] with the slot order
    of dg_halo_plan: send slot i for a peer is that peer's receive slot i."""

    def __init__(self, peers, slice_doubles: int, device, group=None, transport: str = "device"):
        if transport not in ("device", "host"):
            raise ValueError(f"unknown halo transport {transport!r}")
        self.peers = list(peers)
        self.slice_doubles = slice_doubles
        self.group = group
        self.transport = transport
        n = sum(c for _, _, c in self.peers) * slice_doubles
        self.send = torch.zeros(max(n, 1), dtype=torch.float64, device=device)
        self.recv = torch.zeros(max(n, 1), dtype=torch.float64, device=device)
        if transport == "host":
            pin = torch.device(device).type == "cuda"
            self.send_host = torch.zeros(max(n, 1), dtype=torch.float64, pin_memory=pin)
            self.recv_host = torch.zeros(max(n, 1), dtype=torch.float64, pin_memory=pin)

    def _range(self, offset: int, count: int):
        return slice(offset * self.slice_doubles, (offset + count) * self.slice_doubles)

    def start(self, stream=None):
        """Posts every peer's send and receive; returns the works to wait on.
        With the host transport the send buffer is first copied out on
        ``stream`` (the stream the pack was queued on), which is synchronised."""
        send, recv = self.send, self.recv
        if self.transport == "host":
            with torch.cuda.stream(stream) if stream is not None else _nullctx():
                self.send_host.copy_(self.send, non_blocking=True)
            if stream is not None:
                stream.synchronize()
            elif self.send.is_cuda:
                torch.cuda.current_stream().synchronize()
            send, recv = self.send_host, self.recv_host
        ops = []
        for rank, offset, count in self.peers:
            r = self._range(offset, count)
            ops.append(dist.P2POp(dist.isend, send[r], rank, self.group))
            ops.append(dist.P2POp(dist.irecv, recv[r], rank, self.group))
        return dist.batch_isend_irecv(ops) if ops else []

    def finish(self, works, stream=None):
        """Waits for the exchange; with the host transport the received slices
        are then copied into the device receive buffer on ``stream``."""
        for w in works:
            w.wait()
        if self.transport == "host":
            with torch.cuda.stream(stream) if stream is not None else _nullctx():
                self.recv.copy_(self.recv_host, non_blocking=True)


class _nullctx:
    def __enter__(self):
        return None

    def __exit__(self, *exc):
        return False


class DistributedCase:
    """One rank's slab of a periodic box (dg_partition_periodic_box along
    ``axis``) on ``torch.cuda.current_device()``, stepped with halo exchange
    (``transport`` as for HaloExchange)."""

    def __init__(self, n, x0, length, order: int, axis: int = 2, flux: str = "LaxFriedrichs", gamma: float = 1.4,
                 gas_constant: float = 287.05, precision: str = "fp64", group=None, rotate_seed: int = 0,
                 transport: str = "device"):
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.device = torch.cuda.current_device()
        self.mesh, self.part = dg_b200.partition_periodic_box(n, x0, length, self.size, self.rank, axis, rotate_seed)
        self.case = dg_b200.Case(self.mesh, order, flux=flux, gamma=gamma, gas_constant=gas_constant,
                                 precision=precision, device=self.device, part=self.part)
        self.exchange = HaloExchange(self.case.halo_peers(), self.case.halo_slice_doubles(),
                                     torch.device("cuda", self.device), group, transport)
        self.stream = torch.cuda.ExternalStream(self.case.stream_ptr(), device=self.device)

    @property
    def global_elem(self) -> np.ndarray:
        return self.part.global_elem[:self.part.nowned]

    def cfl_time_step(self, Uc: np.ndarray, cfl: float) -> float:
        """The smallest CFL time step over all ranks."""
        dev = torch.device("cuda", self.device) if self.exchange.transport == "device" else "cpu"
        dt = torch.tensor([self.case.cfl_time_step(Uc, cfl)], dtype=torch.float64, device=dev)
        dist.all_reduce(dt, op=dist.ReduceOp.MIN, group=self.group)
        return float(dt.item())

    def _sum_over_ranks(self, values) -> np.ndarray:
        dev = torch.device("cuda", self.device) if self.exchange.transport == "device" else "cpu"
        t = torch.tensor(list(values), dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()

    def l2_error(self, name: str, data=(), t: float = 0.0) -> np.ndarray:
        """Volume-normalised L2 error over the whole decomposed mesh: each
        rank's sum of squares over its owned elements and its volume, summed
        over the ranks (get_error with its MPI_Allreduce, src/post/main.cpp:30-201)."""
        e = self.case.l2_error(name, data, t)
        v = self.case.total_volume()
        s = self._sum_over_ranks([*(e * e * v), v])
        return np.sqrt(s[:5] / s[5])

    def kinetic_energy(self) -> float:
        """Volume-averaged kinetic energy over the whole decomposed mesh."""
        v = self.case.total_volume()
        s = self._sum_over_ranks([self.case.kinetic_energy() * v, v])
        return float(s[0] / s[1])

    def stage(self, s: int, dt: float):
        buf = dg_b200.STAGE_INPUT[s]
        if not self.exchange.peers:
            self.case.rk4_stage(s, dt, 0)
            return
        self.case.halo_pack(buf, self.exchange.send.data_ptr())
        works = self.exchange.start(self.stream)
        self.case.rk4_stage(s, dt, 1)           # interior elements, while the slices travel
        self.exchange.finish(works, self.stream)
        self.case.halo_unpack(buf, self.exchange.recv.data_ptr())
        self.case.rk4_stage(s, dt, 2)           # elements next to a ghost

    def rk4(self, dt: float, nsteps: int):
        """Queues nsteps RK4 steps on the context's stream (not synchronised)."""
        with torch.cuda.stream(self.stream):
            for _ in range(nsteps):
                for s in (1, 2, 3, 4):
                    self.stage(s, dt)

    def sync(self):
        self.stream.synchronize()

    def close(self):
        """Releases the exchange buffers, then the context.  The order matters
        with the host transport: the pinned buffers were copied on the
        context's stream, and torch's pinned-memory allocator records an event
        on that stream when it frees them, so they go while it still exists."""
        if getattr(self, "case", None) is None:
            return
        self.stream.synchronize()
        self.exchange = None
        self.stream = None
        self.case.close()
        self.case = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
