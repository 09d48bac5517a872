"""Domain decomposition: slab partitions with ghost elements, the halo plan,
the exchange over torch.distributed, and (on one GPU) two ranks whose stage
launches and exchanges are ordered by the host.

Bar: every element owned exactly once; every ghost names its owner and its
local id there; send slot i of a rank for a peer is the peer's receive slot i
(same global element and face); after an exchange over gloo every ghost slice
holds its owner's coefficients; on the GPU the owned states of the ranks
match one context over the whole mesh to 1e-13 relative L2 per variable.  (Not
bit for bit: an affine geometry class takes the Jacobian of the first element
met in it, and the elements of a uniform box differ in the last bit of their
node-coordinate differences, so a rank's numbering can pick another
representative.  With one rank the numbering is the global one and the match
is exact.)
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import dg_b200

N = (3, 2, 6)
X0 = (0.0, 0.0, 0.0)
L = (10.0, 10.0, 10.0)
VORTEX_XY = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]


def slice_index(n, f, b0, b1):
    """Coefficient index of boundary-slice entry (b0, b1) of face f (x fastest)."""
    ax = 0 if f in (2, 4) else (1 if f in (1, 3) else 2)
    s = n - 1 if f in (2, 3, 5) else 0
    if ax == 0:
        return b1 * n * n + b0 * n + s
    if ax == 1:
        return b1 * n * n + s * n + b0
    return s * n * n + b1 * n + b0


def parts(nparts, axis=2, seed=0):
    return [dg_b200.partition_periodic_box(N, X0, L, nparts, r, axis, seed) for r in range(nparts)]


@pytest.mark.parametrize("nparts,axis,seed", [(2, 2, 0), (3, 2, 7), (2, 0, 0), (6, 2, 3)])
def test_partition_owns_every_element_once_and_ghosts_name_their_owner(nparts, axis, seed):
    ps = parts(nparts, axis, seed)
    owned = np.concatenate([p.global_elem[:p.nowned] for _, p in ps])
    assert sorted(owned.tolist()) == list(range(N[0] * N[1] * N[2]))
    full = dg_b200.periodic_box(N, X0, L, rotate_seed=seed)
    for mesh, p in ps:
        assert 0 <= p.ninterior <= p.nowned
        for g, (r, le) in enumerate(zip(p.ghost_rank, p.ghost_elem)):
            gid = p.global_elem[p.nowned + g]
            assert r != p.rank and ps[r][1].global_elem[le] == gid
        # local elements carry the global element's node coordinates
        for l, gid in enumerate(p.global_elem):
            assert np.array_equal(mesh.node_coords[mesh.elem_to_node_ids[l]],
                                  full.node_coords[full.elem_to_node_ids[gid]])
        # interior elements have no ghost neighbour; rank columns name owners
        f = mesh.interior_faces
        owner = np.concatenate([np.full(p.nowned, p.rank), p.ghost_rank])
        assert np.array_equal(f[:, 0], owner[f[:, 1]]) and np.array_equal(f[:, 4], owner[f[:, 5]])
        for row in f:
            ghost_side = row[1] >= p.nowned or row[5] >= p.nowned
            if ghost_side:
                assert min(row[1], row[5]) >= p.ninterior


@pytest.mark.parametrize("nparts", [2, 3, 6])
def test_halo_plans_match_between_peers(nparts):
    ps = parts(nparts, seed=5)
    plans = [dg_b200.halo_plan(m, p) for m, p in ps]
    for r, (peers, send, recv) in enumerate(plans):
        gl = ps[r][1].global_elem
        for q, off, cnt in peers:
            qpeers, qsend, qrecv = plans[q]
            (qoff, qcnt), = [(o, c) for rr, o, c in qpeers if rr == r]
            assert qcnt == cnt
            mine = np.stack([gl[send[off:off + cnt, 0]], send[off:off + cnt, 1]], 1)
            gq = ps[q][1].global_elem
            theirs = np.stack([gq[qrecv[qoff:qoff + cnt, 0]], qrecv[qoff:qoff + cnt, 1]], 1)
            assert np.array_equal(mine, theirs)


def test_single_part_has_no_halo():
    (mesh, p), = parts(1)
    assert p.nowned == mesh.nelem and p.ninterior == p.nowned
    assert dg_b200.halo_plan(mesh, p)[0] == []


def test_partition_rejects_bad_arguments():
    with pytest.raises(dg_b200.DGError):
        dg_b200.partition_periodic_box(N, X0, L, 7, 0, 2)   # more parts than layers
    with pytest.raises(dg_b200.DGError):
        dg_b200.partition_periodic_box(N, X0, L, 2, 2, 2)   # part out of range


# ---------------------------------------------------------------- gloo

def _field(gid, n):
    """A coefficient field that identifies its element: [5][n^3]."""
    b = np.arange(n ** 3)
    return np.stack([gid * 1000.0 + v * 100.0 + b for v in range(5)])


def _exchange_worker(rank, world, port, order, transport, errq):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
        import dg_dist
        n = order + 1
        mesh, part = dg_b200.partition_periodic_box(N, X0, L, world, rank, 2, 11)
        peers, send, recv = dg_b200.halo_plan(mesh, part)
        U = np.full((mesh.nelem, 5, n ** 3), np.nan)
        for l in range(part.nowned):
            U[l] = _field(part.global_elem[l], n)
        sd = 5 * n * n
        ex = dg_dist.HaloExchange(peers, sd, "cpu", transport=transport)
        for i, (e, f) in enumerate(send):
            idx = [slice_index(n, f, b0, b1) for b1 in range(n) for b0 in range(n)]
            ex.send[i * sd:(i + 1) * sd] = torch.from_numpy(U[e][:, idx].reshape(-1))
        ex.finish(ex.start())
        got = ex.recv.numpy()
        for i, (g, f) in enumerate(recv):
            idx = [slice_index(n, f, b0, b1) for b1 in range(n) for b0 in range(n)]
            U[g][:, idx] = got[i * sd:(i + 1) * sd].reshape(5, n * n)
            want = _field(part.global_elem[g], n)[:, idx]
            assert np.array_equal(U[g][:, idx], want), (rank, i)
        dist.barrier()
        dist.destroy_process_group()
    except Exception as ex:  # reported to the parent
        errq.put(f"rank {rank}: {ex!r}")
        raise


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,order,transport", [(2, 2, "device"), (3, 1, "device"), (2, 3, "host")])
def test_halo_exchange_over_gloo_fills_every_ghost_slice(world, order, transport):
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    mp.start_processes(_exchange_worker, args=(world, _free_port(), order, transport, errq), nprocs=world, join=True,
                       start_method="spawn")
    assert errq.empty()


# ---------------------------------------------------------------- one GPU, two ranks

@pytest.mark.gpu
@pytest.mark.parametrize("nparts,order,flux", [(2, 3, "LaxFriedrichs"), (3, 2, "HLLC")])
def test_partitioned_ranks_match_one_context(nparts, order, flux):
    """The ranks' contexts share one GPU; each stage the host packs every rank,
    copies the slices between the ranks' buffers, unpacks and launches (no
    kernel waits on another)."""
    full_mesh = dg_b200.periodic_box(N, X0, L, rotate_seed=9)
    full = dg_b200.Case(full_mesh, order, flux=flux, gas_constant=1.0)
    U = full.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = full.cfl_time_step(U, 0.1)
    full.rk4(dt, 3)
    ranks = []
    for r in range(nparts):
        mesh, part = dg_b200.partition_periodic_box(N, X0, L, nparts, r, 2, 9)
        case = dg_b200.Case(mesh, order, flux=flux, gas_constant=1.0, part=part)
        case.set_state(U[part.global_elem[:part.nowned]])
        peers = case.halo_peers()
        n = sum(c for _, _, c in peers) * case.halo_slice_doubles()
        ranks.append((case, part, peers, torch.zeros(max(n, 1), dtype=torch.float64, device="cuda"),
                      torch.zeros(max(n, 1), dtype=torch.float64, device="cuda")))
    sd = ranks[0][0].halo_slice_doubles()
    for _ in range(3):
        for s in (1, 2, 3, 4):
            buf = dg_b200.STAGE_INPUT[s]
            for case, _, _, send, _ in ranks:
                case.halo_pack(buf, send.data_ptr())
                case.sync()
            for r, (case, _, peers, _, recv) in enumerate(ranks):
                for q, off, cnt in peers:
                    (qoff, _), = [(o, c) for rr, o, c in ranks[q][2] if rr == r]
                    recv[off * sd:(off + cnt) * sd].copy_(ranks[q][3][qoff * sd:(qoff + cnt) * sd])
            torch.cuda.synchronize()
            for case, _, _, _, recv in ranks:
                case.halo_unpack(buf, recv.data_ptr())
                case.rk4_stage(s, dt, 1)
                case.rk4_stage(s, dt, 2)
                case.sync()
    want = full.get_state()
    for case, part, *_ in ranks:
        got, ref = case.get_state().reshape(-1, 5), want[part.global_elem[:part.nowned]].reshape(-1, 5)
        nb = np.linalg.norm(ref, axis=0)
        den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())  # rho w is zero in exact arithmetic
        assert (np.linalg.norm(got - ref, axis=0) / den).max() < 1e-13
        assert case.status() == 0


def _nccl_single_rank_worker(rank, port, errq):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        torch.cuda.set_device(0)
        dist.init_process_group("nccl", rank=0, world_size=1, timeout=__import__("datetime").timedelta(seconds=120))
        import dg_dist
        dc = dg_dist.DistributedCase(N, X0, L, 2, gas_constant=1.0)
        U = dc.case.project_ic("IsentropicVortexXY", VORTEX_XY)
        dt = dc.cfl_time_step(U, 0.1)
        dc.rk4(dt, 2)
        dc.sync()
        full = dg_b200.Case(dg_b200.periodic_box(N, X0, L), 2, gas_constant=1.0)
        full.set_state(U)
        full.rk4(dt, 2)
        assert np.array_equal(dc.case.get_state(), full.get_state()[dc.global_elem])
        dist.destroy_process_group()
    except Exception as ex:
        errq.put(repr(ex))
        raise


@pytest.mark.gpu
def test_distributed_case_on_one_rank_matches_one_context():
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    mp.start_processes(_nccl_single_rank_worker, args=(_free_port(), errq), nprocs=1, join=True, start_method="spawn")
    assert errq.empty()


def _host_transport_worker(rank, world, port, order, flux, errq):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        torch.cuda.set_device(0)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=120))
        import dg_dist
        dc = dg_dist.DistributedCase(N, X0, L, order, flux=flux, gas_constant=1.0, rotate_seed=9, transport="host")
        full = dg_b200.Case(dg_b200.periodic_box(N, X0, L, rotate_seed=9), order, flux=flux, gas_constant=1.0)
        U = full.project_ic("IsentropicVortexXY", VORTEX_XY)
        dc.case.set_state(U[dc.global_elem])
        dt = dc.cfl_time_step(dc.case.get_state(), 0.1)
        dc.rk4(dt, 3)
        dc.sync()
        full.rk4(dt, 3)
        got, ref = dc.case.get_state().reshape(-1, 5), full.get_state()[dc.global_elem].reshape(-1, 5)
        nb = np.linalg.norm(ref, axis=0)
        den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())  # rho w is zero in exact arithmetic
        d = (np.linalg.norm(got - ref, axis=0) / den).max()
        assert d < 1e-13, (rank, d)
        assert dc.case.status() == 0
        assert dc.exchange.peers, "every rank of a periodic slab decomposition has peers"
        # the error and kinetic energy summed over the ranks are the whole mesh's
        np.testing.assert_allclose(dc.l2_error("IsentropicVortexXY", VORTEX_XY, 3 * dt),
                                   full.l2_error("IsentropicVortexXY", VORTEX_XY, 3 * dt), rtol=1e-11, atol=1e-14)
        assert abs(dc.kinetic_energy() / full.kinetic_energy() - 1.0) < 1e-12
        dc.close()
        full.close()
        dist.barrier()
        dist.destroy_process_group()
    except Exception as ex:
        errq.put(f"rank {rank}: {ex!r}")
        raise


@pytest.mark.gpu
@pytest.mark.parametrize("world,order,flux", [(2, 3, "LaxFriedrichs"), (3, 2, "HLLC")])
def test_distributed_case_ranks_step_with_host_transport(world, order, flux):
    """DistributedCase.stage as it runs between GPUs -- pack, exchange started,
    interior launch overlapping it, wait, unpack, boundary launch, all ordered
    on each rank's stream -- with world processes on one GPU exchanging over
    gloo through pinned host buffers (no kernel waits on another rank); every
    rank's owned state matches one context over the whole mesh."""
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    mp.start_processes(_host_transport_worker, args=(world, _free_port(), order, flux, errq), nprocs=world,
                       join=True, start_method="spawn")
    assert errq.empty(), errq.get()
