"""Batched ensembles (dg_batch_*): independent cases of different order, mesh
size and time step advanced by one graph of per-order stage launches.

Bar: each case of a batch is bit-identical to a single-case context running
the same stage variant on the same case (the per-case time step enters the
update as dt * dtf with dt = 1 in the batch and dtf = 1 in a context, the same
product), and a small batched case matches the CPU oracle to 1e-12 relative
L2 per variable.
"""
import numpy as np
import pytest

import dg_b200
import pyoracle

VORTEX_XY = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]

# (mesh cells, rotation seed, order): mixed orders, repeated orders (groups of
# several cases), anisotropic boxes and rotated element numberings
CASES = [((3, 3, 2), 17, 2), ((2, 2, 2), 0, 1), ((4, 2, 3), 5, 3), ((2, 3, 2), 9, 2), ((2, 2, 2), 3, 5),
         ((3, 2, 2), 0, 4), ((2, 2, 3), 0, 0), ((3, 3, 3), 21, 3)]


def vortex(i):
    rng = np.random.default_rng(100 + i)
    beta = rng.uniform(1, 5)
    xc, yc = rng.uniform(3, 7, 2)
    u, v = rng.uniform(0.5, 1.5, 2)
    return [1.0, u, v, 1.0, beta, xc, yc, 10.0, 10.0]


def rel_l2(a, b):
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    nb = np.linalg.norm(b, axis=0)
    den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())
    return np.linalg.norm(a - b, axis=0) / den


def meshes():
    return [dg_b200.periodic_box(n, (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=s) for n, s, _ in CASES]


# ---------------------------------------------------------------- host side

def test_batch_rejects_bad_cases_before_touching_the_device():
    ms = meshes()
    with pytest.raises(dg_b200.DGError, match="case 1: order must be 0..5"):
        dg_b200.Batch([(ms[0], 2), (ms[1], 7)])
    open_mesh = dg_b200.Mesh(ms[1].node_coords, ms[1].elem_to_node_ids, ms[1].interior_faces[:-1])
    with pytest.raises(dg_b200.DGError, match="case 1:") as ei:
        dg_b200.Batch([(ms[0], 2), (open_mesh, 2)])
    assert ei.value.code in (1, 5)


def test_batch_create_without_gpu_fails_loudly():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(dg_b200.DGError, match="DG_ERR_CUDA"):
        dg_b200.Batch([(m, p) for m, (_, _, p) in zip(meshes(), CASES)])


# ---------------------------------------------------------------- GPU

def setup_pair(precision="fp64", cfl=0.1):
    ms = meshes()
    batch = dg_b200.Batch([(m, p) for m, (_, _, p) in zip(ms, CASES)], gas_constant=1.0, precision=precision)
    singles, U0, dts = [], [], []
    for i, (m, (_, _, p)) in enumerate(zip(ms, CASES)):
        case = dg_b200.Case(m, p, gas_constant=1.0, precision=precision)
        U = case.project_ic("IsentropicVortexXY", vortex(i))
        Ub = batch.project_ic(i, "IsentropicVortexXY", vortex(i))
        assert np.array_equal(U, Ub)
        dt = batch.cfl_time_step(i, Ub, cfl)
        assert dt == case.cfl_time_step(U, cfl)
        batch.set_time_step(i, dt)
        singles.append(case)
        U0.append(U)
        dts.append(dt)
    return batch, singles, U0, dts


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
def test_batch_cases_bit_identical_to_single_contexts(precision):
    batch, singles, U0, dts = setup_pair(precision)
    groups = batch.groups()
    assert sorted(g[0] for g in groups) == sorted(set(p for _, _, p in CASES))
    assert sum(g[1] for g in groups) == len(CASES)
    batch.rk4(4)
    for i, case in enumerate(singles):
        case.rk4(dts[i], 4)
        assert np.array_equal(batch.get_state(i), case.get_state()), i
    assert batch.status() == 0


@pytest.mark.gpu
def test_batched_case_matches_oracle():
    batch, singles, U0, dts = setup_pair()
    batch.rk4(5)
    for i in (0, 4):  # p = 2 on a rotated mesh, p = 5
        n, seed, p = CASES[i]
        mesh = dg_b200.periodic_box(n, (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=seed)
        orc = pyoracle.OracleCase.from_mesh(mesh, p, gas_constant=1.0)
        U_orc = orc.rk4(U0[i], dts[i], 5)
        assert rel_l2(batch.get_state(i), U_orc).max() < 1e-12


@pytest.mark.gpu
def test_batch_error_tuning_and_zero_time_step():
    batch, singles, U0, dts = setup_pair()
    batch.set_time_step(1, 0.0)      # case 1 does not move
    batch.tune(reps=1)
    ms = batch.rk4_timed(3)
    assert ms > 0
    assert np.array_equal(batch.get_state(1), U0[1])
    t = 3 * dts[0]
    for i in (0, 2):
        case = singles[i]
        # the tuned variant of the case's group, on the single context too
        case.stage_variant = [g for g in batch.groups() if g[0] == CASES[i][2]][0][3]
        case.rk4(dts[i], 3)
        assert np.array_equal(batch.get_state(i), case.get_state())
        e_b = batch.l2_error(i, "IsentropicVortexXY", vortex(i), 3 * dts[i])
        e_s = case.l2_error("IsentropicVortexXY", vortex(i), 3 * dts[i])
        assert np.allclose(e_b, e_s, rtol=1e-12, atol=0)
    assert t > 0


# ---------------------------------------------------------------- one launch per RK stage

ENS = [c for c in CASES if c[2] > 0]  # orders 1..5: the ensemble launch takes every group


def setup_ensemble(precision):
    ms = [dg_b200.periodic_box(n, (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=s) for n, s, _ in ENS]
    batch = dg_b200.Batch([(m, p) for m, (_, _, p) in zip(ms, ENS)], gas_constant=1.0, precision=precision)
    singles, dts = [], []
    for i, (m, (_, _, p)) in enumerate(zip(ms, ENS)):
        case = dg_b200.Case(m, p, gas_constant=1.0, precision=precision)
        U = case.project_ic("IsentropicVortexXY", vortex(i))
        Ub = batch.project_ic(i, "IsentropicVortexXY", vortex(i))
        dt = batch.cfl_time_step(i, Ub, 0.1)
        batch.set_time_step(i, dt)
        singles.append(case)
        dts.append(dt)
    return batch, singles, dts


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
def test_single_launch_batch_bit_identical_to_single_contexts(precision):
    """Orders 1..5 in one launch per RK stage (plus one face launch): every case
    bit-identical to a single context running its group's variant (a compiled
    128-thread variant of the order), then the same after switching the batch
    to one launch per group."""
    batch, singles, dts = setup_ensemble(precision)
    assert not batch.single_launch  # the default: one launch per group
    batch.single_launch = True
    variant = {g[0]: g[3] for g in batch.groups()}
    for i, case in enumerate(singles):
        case.stage_variant = variant[ENS[i][2]]
        assert case.stage_variants()[variant[ENS[i][2]]][1] == 128
    batch.rk4(3)
    for i, case in enumerate(singles):
        case.rk4(dts[i], 3)
        assert np.array_equal(batch.get_state(i), case.get_state()), i
    assert batch.status() == 0
    # back to one launch per group: each group's own (default) variant
    batch.single_launch = False
    assert not batch.single_launch
    variant = {g[0]: g[3] for g in batch.groups()}
    batch.rk4(2)
    for i, case in enumerate(singles):
        case.stage_variant = variant[ENS[i][2]]
        case.rk4(dts[i], 2)
        assert np.array_equal(batch.get_state(i), case.get_state()), i


@pytest.mark.gpu
def test_single_launch_batch_matches_oracle_and_rejects_order_zero():
    batch, singles, dts = setup_ensemble("fp64")
    batch.single_launch = True
    U0 = [s.get_state() for s in singles]
    batch.rk4(4)
    for i in (0, 3):  # p = 2 on a rotated mesh, p = 5
        n, seed, p = ENS[i]
        mesh = dg_b200.periodic_box(n, (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=seed)
        orc = pyoracle.OracleCase.from_mesh(mesh, p, gas_constant=1.0)
        assert rel_l2(batch.get_state(i), orc.rk4(U0[i], dts[i], 4)).max() < 1e-12
    # a batch with an order-0 group runs one launch per group and refuses the single launch
    full, _, _, _ = setup_pair()
    assert not full.single_launch
    with pytest.raises(dg_b200.DGError) as ei:
        full.single_launch = True
    assert ei.value.code == 5


@pytest.mark.gpu
def test_batch_tuner_keeps_the_faster_launch_mode_and_the_state():
    batch, singles, dts = setup_ensemble("mixed_fp32")
    before = [batch.get_state(i) for i in range(len(ENS))]
    batch.tune(reps=1)
    assert all(np.array_equal(batch.get_state(i), u) for i, u in enumerate(before))
    mode = batch.single_launch
    variant = {g[0]: g[3] for g in batch.groups()}
    batch.rk4(2)
    for i, case in enumerate(singles):
        case.stage_variant = variant[ENS[i][2]]
        case.rk4(dts[i], 2)
        assert np.array_equal(batch.get_state(i), case.get_state()), (i, mode)
