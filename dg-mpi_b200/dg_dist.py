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

    def __init__(self, peers, slice_doubles: int, device, group=None):
        self.peers = list(peers)
        self.slice_doubles = slice_doubles
        self.group = group
        n = sum(c for _, _, c in self.peers) * slice_doubles
        self.send = torch.zeros(max(n, 1), dtype=torch.float64, device=device)
        self.recv = torch.zeros(max(n, 1), dtype=torch.float64, device=device)

    def _range(self, offset: int, count: int):
        return slice(offset * self.slice_doubles, (offset + count) * self.slice_doubles)

    def start(self):
        """Posts every peer's send and receive; returns the works to wait on."""
        ops = []
        for rank, offset, count in self.peers:
            r = self._range(offset, count)
            ops.append(dist.P2POp(dist.isend, self.send[r], rank, self.group))
            ops.append(dist.P2POp(dist.irecv, self.recv[r], rank, self.group))
        return dist.batch_isend_irecv(ops) if ops else []


class DistributedCase:
    """One rank's slab of a periodic box (dg_partition_periodic_box along
    ``axis``) on ``torch.cuda.current_device()``, stepped with halo exchange."""

    def __init__(self, n, x0, length, order: int, axis: int = 2, flux: str = "LaxFriedrichs", gamma: float = 1.4,
                 gas_constant: float = 287.05, precision: str = "fp64", group=None, rotate_seed: int = 0):
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.device = torch.cuda.current_device()
        self.mesh, self.part = dg_b200.partition_periodic_box(n, x0, length, self.size, self.rank, axis, rotate_seed)
        self.case = dg_b200.Case(self.mesh, order, flux=flux, gamma=gamma, gas_constant=gas_constant,
                                 precision=precision, device=self.device, part=self.part)
        self.exchange = HaloExchange(self.case.halo_peers(), self.case.halo_slice_doubles(),
                                     torch.device("cuda", self.device), group)
        self.stream = torch.cuda.ExternalStream(self.case.stream_ptr(), device=self.device)

    @property
    def global_elem(self) -> np.ndarray:
        return self.part.global_elem[:self.part.nowned]

    def cfl_time_step(self, Uc: np.ndarray, cfl: float) -> float:
        """The smallest CFL time step over all ranks."""
        dt = torch.tensor([self.case.cfl_time_step(Uc, cfl)], dtype=torch.float64,
                          device=torch.device("cuda", self.device))
        dist.all_reduce(dt, op=dist.ReduceOp.MIN, group=self.group)
        return float(dt.item())

    def stage(self, s: int, dt: float):
        buf = dg_b200.STAGE_INPUT[s]
        if not self.exchange.peers:
            self.case.rk4_stage(s, dt, 0)
            return
        self.case.halo_pack(buf, self.exchange.send.data_ptr())
        works = self.exchange.start()
        self.case.rk4_stage(s, dt, 1)           # interior elements, while the slices travel
        for w in works:
            w.wait()
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
