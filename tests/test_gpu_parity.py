"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bar (FP64 path): relative L2 difference per conserved variable <= 1e-12 after
time stepping, <= 1e-11 for a single residual evaluation (a difference of
volume and surface terms), bit-exact for size-independent identities.  A
variable that is identically zero in exact arithmetic (rho v of the x-z
vortex, rho w of the x-y vortex) is normalised by the largest variable's norm.
"""
import numpy as np
import pytest

import dg_b200
import pyoracle

pytestmark = pytest.mark.gpu

VORTEX_XY = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]  # rho, u, v, p, beta, xc, yc, Lx, Ly


def rel_l2(a, b):
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    nb = np.linalg.norm(b, axis=0)
    # a variable below 1e-3 of the largest norm is zero in exact arithmetic:
    # measure it against the largest variable's norm
    den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())
    return np.linalg.norm(a - b, axis=0) / den


def make_pair(n, p, flux="LaxFriedrichs", rotate_seed=0, length=(10.0, 10.0, 10.0), gas_constant=1.0):
    mesh = dg_b200.periodic_box(n, (0.0, 0.0, 0.0), length, rotate_seed=rotate_seed)
    gpu = dg_b200.Case(mesh, p, flux=flux, gas_constant=gas_constant)
    orc = pyoracle.OracleCase.from_mesh(mesh, p, flux=flux, gas_constant=gas_constant)
    return mesh, gpu, orc


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
@pytest.mark.parametrize("p", [0, 1, 2, 3, 4, 5])
def test_residual_matches_oracle(p, flux):
    _, gpu, orc = make_pair((3, 2, 2), p, flux=flux, rotate_seed=11)
    U = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    gpu.set_state(U)
    R_gpu = gpu.residual()
    R_orc = orc.residual(U)
    assert rel_l2(R_gpu, R_orc).max() < 1e-11, rel_l2(R_gpu, R_orc)
    assert gpu.status() == 0


@pytest.mark.parametrize("p", [1, 3])
def test_residual_on_unrotated_and_single_element_meshes(p):
    for n in [(1, 1, 1), (2, 1, 3), (4, 4, 4)]:
        mesh = dg_b200.periodic_box(n, (0, 0, 0), (1, 1, 1))
        gpu = dg_b200.Case(mesh, p, flux="HLLC", gas_constant=1.0)
        orc = pyoracle.OracleCase.from_mesh(mesh, p, flux="HLLC", gas_constant=1.0)
        U = orc.project_ic("IsentropicVortex")
        gpu.set_state(U)
        assert rel_l2(gpu.residual(), orc.residual(U)).max() < 1e-11


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_mass_inverse_residual_matches_oracle(p):
    _, gpu, orc = make_pair((2, 3, 2), p, rotate_seed=5)
    U = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    gpu.set_state(U)
    dt = 1e-3
    dU_gpu = gpu.mass_inverse_residual(dt)
    dU_orc = orc.fe(U, dt, 1) - U
    assert rel_l2(dU_gpu, dU_orc).max() < 1e-10


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_rk4_steps_match_oracle(p, flux):
    _, gpu, orc = make_pair((3, 3, 2), p, flux=flux, rotate_seed=17)
    U = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = gpu.cfl_time_step(U, 0.1)
    gpu.set_state(U)
    gpu.rk4(dt, 5)
    U_orc = orc.rk4(U, dt, 5)
    assert rel_l2(gpu.get_state(), U_orc).max() < 1e-12


def test_forward_euler_matches_oracle():
    _, gpu, orc = make_pair((2, 2, 2), 2, rotate_seed=2)
    U = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = gpu.cfl_time_step(U, 0.05)
    gpu.set_state(U)
    gpu.fe(dt, 3)
    gpu.rk4(dt, 1)  # the RK4 graph is rebuilt after the FE buffer swap
    U_orc = orc.rk4(orc.fe(U, dt, 3), dt, 1)
    assert rel_l2(gpu.get_state(), U_orc).max() < 1e-12


def test_config_vortex_8cubed_p2_100_steps():
    """The CPU-runnable configuration: [0,10]^3, 8^3 elements, p=2, x-y
    vortex (beta 5, centre (5,5), u=(1,1,0)), default Lax-Friedrichs flux,
    RK4 at CFL 0.1 for 100 steps; GPU vs oracle and both vs the exact
    advected vortex."""
    _, gpu, orc = make_pair((8, 8, 8), 2)
    U0 = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = gpu.cfl_time_step(U0, 0.1)
    gpu.set_state(U0)
    gpu.rk4(dt, 100)
    U_orc = orc.rk4(U0, dt, 100)
    U_gpu = gpu.get_state()
    assert rel_l2(U_gpu, U_orc).max() < 1e-12
    t = 100 * dt
    e_gpu = gpu.l2_error("IsentropicVortexXY", VORTEX_XY, t)
    e_orc = orc.l2_error(U_orc, "IsentropicVortexXY", VORTEX_XY, t)
    np.testing.assert_allclose(e_gpu[[0, 1, 2, 4]], e_orc[[0, 1, 2, 4]], rtol=1e-9)
    assert e_gpu[0] < 5e-2  # the scheme tracks the exact solution


def test_vortex3d_regression_on_gpu(golden):
    g = golden["vortex3d_regression"]
    mesh = dg_b200.periodic_box((4, 4, 4), (0, 0, 0), (1, 1, 1))
    gpu = dg_b200.Case(mesh, g["order"], flux=g["flux"], gamma=g["gamma"], gas_constant=g["gas_constant"])
    gpu.project_ic("IsentropicVortex")
    gpu.rk4(g["timestep"], int(g["end"] / g["timestep"]))
    err = gpu.l2_error("IsentropicVortex")
    ref = np.array(g["l2_errors"])
    for s in (0, 1, 3, 4):
        assert abs(err[s] - ref[s]) <= 1e-12 * ref[s], (s, err[s], ref[s])
    assert err[2] < 1e-13
    assert gpu.status() == 0


@pytest.mark.parametrize("p", [0, 1, 2, 3, 4, 5])
def test_initial_projection_and_error_match_oracle(p):
    """The on-device L2 projection (one CTA per element) against the oracle's."""
    _, gpu, orc = make_pair((2, 2, 3), p, rotate_seed=9)
    U_gpu = gpu.project_ic("IsentropicVortexXY", VORTEX_XY)
    U_orc = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    assert rel_l2(U_gpu, U_orc).max() < 1e-13
    tg_gpu = gpu.project_ic("TaylorGreen", [0.1])
    tg_orc = orc.project_ic("TaylorGreen", [0.1])
    assert rel_l2(tg_gpu, tg_orc).max() < 1e-13
    gpu.project_ic("IsentropicVortexXY", VORTEX_XY)
    e_gpu = gpu.l2_error("IsentropicVortexXY", VORTEX_XY, 0.3)
    e_orc = orc.l2_error(U_orc, "IsentropicVortexXY", VORTEX_XY, 0.3)
    np.testing.assert_allclose(e_gpu[[0, 1, 2, 4]], e_orc[[0, 1, 2, 4]], rtol=1e-10)
    assert abs(gpu.total_volume() - orc.total_volume()) < 1e-12 * orc.total_volume()


@pytest.mark.parametrize("p", [1, 3, 5])
def test_free_stream_preservation(p):
    mesh = dg_b200.periodic_box((3, 2, 2), (0, 0, 0), (1.0, 0.7, 2.0), rotate_seed=4)
    gpu = dg_b200.Case(mesh, p, flux="HLLC")
    U = gpu.project_ic("Uniform", [1.2, 0.3, -0.2, 0.1, 2.5])
    R = gpu.residual()
    assert np.abs(R).max() < 1e-12
    gpu.rk4(1e-3, 3)
    assert np.abs(gpu.get_state() - U).max() < 1e-13


def test_conservation_and_translation_invariance_at_full_size():
    """64^3 elements, p=3 (the at-scale configuration): the residual sums to
    zero over the periodic box, and translating the state by one element
    translates the residual bit-for-bit (the periodic gather at full size)."""
    n = 64
    mesh = dg_b200.periodic_box((n, n, n), (0, 0, 0), (10.0, 10.0, 10.0))
    gpu = dg_b200.Case(mesh, 3, gas_constant=1.0)
    U = gpu.project_ic("IsentropicVortexXY", VORTEX_XY)
    R = gpu.residual()
    total = R.sum(axis=(0, 1))
    assert np.all(np.abs(total) < 1e-12 * np.abs(R).sum(axis=(0, 1)).max())
    shifted = np.roll(U.reshape(n, n, n, -1, 5), 1, axis=2).reshape(U.shape)  # +1 element in x
    gpu.set_state(shifted)
    R2 = gpu.residual()
    np.testing.assert_array_equal(R2, np.roll(R.reshape(n, n, n, -1, 5), 1, axis=2).reshape(R.shape))
    del R, R2
    # two RK4 steps at full size keep the state finite and the status clean
    gpu.set_state(U)
    gpu.rk4(gpu.cfl_time_step(U, 0.1), 2)
    assert gpu.status() == 0


def test_config_64cubed_p3_rk4_steps_match_oracle():
    """The at-scale FP64 configuration against the CPU oracle (the reference's
    dense per-element algorithm): 64^3 elements of [0,10]^3, p = 3, x-y vortex,
    Lax-Friedrichs, RK4 at CFL 0.1, two steps from the same projected state,
    <= 1e-12 relative L2 per variable (src/solver/base.cpp:402-413 stepped by
    src/numerics/timestepping/stepper.cpp:72-142).  The oracle holds the
    reference's dense inverse mass matrices and per-point geometry (~30 GB of
    host memory at 64^3, ~1 minute on 16 cores); a host with less memory runs
    the same case at 48^3."""
    import psutil

    n = 64 if psutil.virtual_memory().available > 48e9 else 48
    _, gpu, orc = make_pair((n, n, n), 3)
    U0 = gpu.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = gpu.cfl_time_step(U0, 0.1)
    gpu.rk4(dt, 2)
    U_gpu = gpu.get_state()
    U_orc = orc.rk4(U0, dt, 2)
    d = rel_l2(U_gpu, U_orc)
    print(f"{n}^3 p=3 two RK4 steps: GPU vs oracle relative L2 {d}")
    assert d.max() < 1e-12, d
    assert gpu.status() == 0


def test_nonphysical_state_is_reported_not_faulted():
    mesh = dg_b200.periodic_box((2, 2, 2))
    gpu = dg_b200.Case(mesh, 1, flux="HLLC")
    U = gpu.project_ic("Uniform", [1.0, 0.1, 0.0, 0.0, 2.5])
    U[3, :, 0] = -1.0  # negative density in one element
    gpu.set_state(U)
    with pytest.raises(dg_b200.DGError) as ei:
        gpu.rk4(1e-3, 1)
    assert ei.value.code == 3
    flags = gpu.status()  # reported flags stay readable until dg_status clears them
    assert flags & 1  # non-positive density
    # the context stays usable
    gpu.project_ic("Uniform", [1.0, 0.1, 0.0, 0.0, 2.5])
    gpu.rk4(1e-3, 1)
    assert gpu.status() == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_garbage_states_are_reported_by_every_default_variant(flux, precision):
    """States no physical flow has (NaN, infinities, negative density or
    energy, huge values) stepped by the default variant of p = 1 .. 5 end in
    DG_ERR_NONPHYSICAL with the status word set, and a valid state steps
    again afterwards: the kernels' arithmetic on garbage reports, it never
    faults or hangs (no index depends on a state value)."""
    rng = np.random.default_rng(23)
    mesh = dg_b200.periodic_box((3, 2, 2), (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=2)
    for p in range(1, 6):
        case = dg_b200.Case(mesh, p, flux=flux, gas_constant=1.0, precision=precision)
        good = case.project_ic("IsentropicVortexXY", VORTEX_XY)
        dt = case.cfl_time_step(good, 0.1)
        for garbage in (np.nan, np.inf, -1.0, 1e300):
            U = good.copy()
            idx = rng.integers(0, U.size, 7)
            U.reshape(-1)[idx] = garbage
            U[0, :, 0] = garbage if garbage != 1e300 else -1.0  # always one bad density
            case.set_state(U)
            with pytest.raises(dg_b200.DGError) as ei:
                case.rk4(dt, 1)
            assert ei.value.code == 3, (p, garbage, ei.value)
            assert case.status() != 0
        case.set_state(good)
        case.rk4(dt, 2)
        assert case.status() == 0
        case.close()


def test_time_step_change_rebuilds_graph():
    _, gpu, orc = make_pair((2, 2, 2), 2)
    U = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    gpu.set_state(U)
    gpu.rk4(1e-3, 2)
    gpu.rk4(2e-3, 2)
    U_orc = orc.rk4(orc.rk4(U, 1e-3, 2), 2e-3, 2)
    assert rel_l2(gpu.get_state(), U_orc).max() < 1e-12


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
@pytest.mark.parametrize("p", [0, 1, 2, 3, 4, 5])
def test_every_stage_variant_matches_oracle(p, flux):
    """Every compiled launch variant (elements and threads per CTA, variable
    groups and the launch options: one-phase groups, single coefficient
    buffer, unfused volume, row-split traces, one flux point per thread) --
    the tuner may pick any of them: FP64 variants against the oracle at 1e-12
    after 3 RK4 steps, mixed-precision variants against the FP64 result at 1e-6."""
    mesh = dg_b200.periodic_box((3, 2, 3), (0.0, 0.0, 0.0), (10.0, 10.0, 10.0), rotate_seed=7)
    orc = pyoracle.OracleCase.from_mesh(mesh, p, flux=flux, gas_constant=1.0)
    U = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    ref = None
    for precision in ("fp64", "mixed_fp32"):
        case = dg_b200.Case(mesh, p, flux=flux, gas_constant=1.0, precision=precision)
        dt = case.cfl_time_step(U, 0.1)
        if ref is None:
            ref = orc.rk4(U, dt, 3)
        for v, info in enumerate(case.stage_variants()):
            if info[3] != precision or "ge" in info[4].split("+"):
                continue  # general-geometry variants run on non-affine meshes (test_gpu_general.py)
            case.stage_variant = v
            case.set_state(U)
            case.rk4(dt, 3)
            tol = 1e-12 if precision == "fp64" else 1e-6
            assert rel_l2(case.get_state(), ref).max() < tol, (precision, v, info)
            assert case.status() == 0
        case.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
def test_chunked_stages_are_bit_identical(precision):
    """RK4 steps with each stage split into element chunks (face launches on a
    second stream beside the previous chunk's stage launch) give the same bits
    as one face and one stage launch per stage, for chunk counts that do and
    do not divide the mesh, on a mesh with rotated elements."""
    mesh = dg_b200.periodic_box((7, 6, 5), (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=9)
    case = dg_b200.Case(mesh, 3, flux="HLLC", gas_constant=1.0, precision=precision)
    fx = [i for i, v in enumerate(case.stage_variants()) if v[3] == precision and "fx" in v[4].split("+")]
    assert fx
    case.stage_variant = fx[0]
    U0 = case.project_ic("IsentropicVortexXY", [1, 1, 1, 1, 5, 5, 5, 10, 10])
    dt = case.cfl_time_step(U0, 0.1)
    case.rk4(dt, 3)
    ref = case.get_state()
    for chunks in (2, 3, 7, 64):
        case.stage_chunks = chunks
        assert case.stage_chunks == chunks
        case.set_state(U0)
        case.rk4(dt, 3)
        assert np.array_equal(case.get_state(), ref), chunks
    case.stage_chunks = 1
    case.set_state(U0)
    case.rk4(dt, 3)
    assert np.array_equal(case.get_state(), ref)
    assert case.status() == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed_fp32"])
@pytest.mark.parametrize("p", [2, 3, 4, 5])
def test_folded_lift_gather_is_bit_identical(p, precision):
    """Launch option MG (the six faces' lifts added inside the inverse mass's
    x pass instead of a pass of their own) performs the same additions in the
    same order: RK4 and forward-Euler steps and the residual give the same
    bits as the variant without it."""
    mesh = dg_b200.periodic_box((7, 6, 5), (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=9)
    case = dg_b200.Case(mesh, p, flux="HLLC", gas_constant=1.0, precision=precision)
    U0 = case.project_ic("IsentropicVortexXY", [1, 1, 1, 1, 5, 5, 5, 10, 10])
    dt = case.cfl_time_step(U0, 0.1)
    vs = case.stage_variants()
    pairs = []
    for i, v in enumerate(vs):
        opts = v[4].split("+")
        if v[3] != precision or "mg" not in opts:
            continue
        base = {o for o in opts if o != "mg" and not o.startswith("mb")}
        j = [k for k, w in enumerate(vs) if w[:4] == v[:4] and "mg" not in w[4].split("+")
             and {o for o in w[4].split("+") if not o.startswith("mb")} == base]
        assert j, v
        pairs.append((i, j[0]))
    assert pairs
    for i, j in pairs:
        got = []
        for k in (i, j):
            case.stage_variant = k
            case.set_state(U0)
            R = case.residual()
            case.rk4(dt, 3)
            case.fe(dt, 1)
            got.append((R, case.get_state()))
        assert np.array_equal(got[0][0], got[1][0]) and np.array_equal(got[0][1], got[1][1]), (vs[i], vs[j])
    assert case.status() == 0


def test_bounded_wait_gives_up_and_the_device_stays_usable():
    """Failure detection without a fault: a bounded device wait on a barrier
    that nothing completes gives up after its limit and reports
    DG_ERR_TIMEOUT; the same wait on a completed barrier returns at once; a
    context created afterwards computes as before."""
    limit = 2_000_000  # SM cycles, about 1 ms
    rc, cycles = dg_b200.probe_bounded_wait(0, limit, arrive=False)
    assert rc == dg_b200.DG_ERR_TIMEOUT and cycles >= limit, (rc, cycles)
    assert "gave up" in dg_b200.library().dg_last_error(None).decode()
    rc, cycles = dg_b200.probe_bounded_wait(0, limit, arrive=True)
    assert rc == dg_b200.DG_OK and cycles < limit, (rc, cycles)
    mesh = dg_b200.periodic_box((3, 2, 3), (0.0, 0.0, 0.0), (10.0, 10.0, 10.0), rotate_seed=7)
    orc = pyoracle.OracleCase.from_mesh(mesh, 2, flux="HLLC", gas_constant=1.0)
    U = orc.project_ic("IsentropicVortexXY", VORTEX_XY)
    case = dg_b200.Case(mesh, 2, flux="HLLC", gas_constant=1.0)
    case.set_state(U)
    assert rel_l2(case.residual(), orc.residual(U)).max() < 1e-11
    assert case.status() == 0
    case.close()
