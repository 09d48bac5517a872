"""Mixed-precision residual (FP32 traces, fluxes and contractions; FP64 state,
residual accumulation, inverse mass and RK update) against the FP64 path.

Bar: relative L2 difference per conserved variable <= 1e-6 after time
stepping (a variable that is identically zero in exact arithmetic is
normalised by the largest variable's norm), and the same L2 error against
the exact advected vortex to within that difference.
"""
import numpy as np
import pytest

import dg_b200

pytestmark = pytest.mark.gpu

VORTEX_XY = [1.0, 1.0, 1.0, 1.0, 5.0, 5.0, 5.0, 10.0, 10.0]
TOL = 1e-6


def rel_l2(a, b):
    a = a.reshape(-1, 5)
    b = b.reshape(-1, 5)
    nb = np.linalg.norm(b, axis=0)
    # a variable below 1e-3 of the largest norm is zero in exact arithmetic:
    # measure it against the largest variable's norm
    den = np.where(nb > 1e-3 * nb.max(), nb, nb.max())
    return np.linalg.norm(a - b, axis=0) / den


@pytest.mark.parametrize("p,n,steps", [(1, 12, 60), (3, 8, 60), (5, 8, 100)])
def test_mixed_matches_fp64_on_vortex(p, n, steps):
    mesh = dg_b200.periodic_box((n, n, n), (0, 0, 0), (10.0, 10.0, 10.0))
    f64 = dg_b200.Case(mesh, p, gas_constant=1.0, precision="fp64")
    mix = dg_b200.Case(mesh, p, gas_constant=1.0, precision="mixed_fp32")
    U0 = f64.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = f64.cfl_time_step(U0, 0.1)
    mix.set_state(U0)
    f64.rk4(dt, steps)
    mix.rk4(dt, steps)
    d = rel_l2(mix.get_state(), f64.get_state())
    assert d.max() < TOL, d
    t = steps * dt
    e64 = f64.l2_error("IsentropicVortexXY", VORTEX_XY, t)
    emx = mix.l2_error("IsentropicVortexXY", VORTEX_XY, t)
    np.testing.assert_allclose(emx[[0, 1, 2, 4]], e64[[0, 1, 2, 4]], rtol=1e-3)
    assert mix.status() == 0


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_mixed_residual_is_fp32_accurate(flux):
    mesh = dg_b200.periodic_box((3, 2, 2), (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=21)
    f64 = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0)
    mix = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0, precision="mixed_fp32")
    U = f64.project_ic("IsentropicVortexXY", VORTEX_XY)
    mix.set_state(U)
    R64, Rmx = f64.residual(), mix.residual()
    # FP32 arithmetic on O(1) fluxes: errors of a few ulp of float relative to the flux scale
    scale = np.abs(R64).max()
    assert np.abs(Rmx - R64).max() < 1e-5 * scale


def test_mixed_free_stream_and_tuner():
    mesh = dg_b200.periodic_box((4, 3, 2), (0, 0, 0), (1.0, 1.0, 1.0), rotate_seed=3)
    mix = dg_b200.Case(mesh, 2, flux="HLLC", precision="mixed_fp32")
    U = mix.project_ic("Uniform", [1.1, 0.2, 0.1, -0.3, 2.6])
    best, ms = mix.tune_stage(reps=1)
    variants = mix.stage_variants()
    assert variants[best][3] == "mixed_fp32"
    # variants of the other precision, and the general-geometry ones (this mesh is affine), are not timed
    assert all((t < 0) == (v[3] != "mixed_fp32" or "ge" in v[4].split("+")) for v, t in zip(variants, ms))
    mix.rk4(1e-3, 5)
    assert np.abs(mix.get_state() - U).max() < 1e-6


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_low_mach_taylor_green_mixed_within_bound(flux):
    """At Mach 0.1 the energy (~180) dwarfs the momenta; the FP32 residual
    works on rE - E_ref, so the momenta keep FP32's digits, with both fluxes
    (HLLC evaluates its pressures in the shifted frame, dgp::flux_hllc_shift)."""
    L = 2 * np.pi
    mesh = dg_b200.periodic_box((8, 8, 8), (0, 0, 0), (L, L, L))
    f64 = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0, precision="fp64")
    mix = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0, precision="mixed_fp32")
    U0 = f64.project_ic("TaylorGreen", [0.1])
    dt = f64.cfl_time_step(U0, 0.1)
    mix.set_state(U0)
    f64.rk4(dt, 40)
    mix.rk4(dt, 40)
    d = rel_l2(mix.get_state(), f64.get_state())
    assert d.max() < TOL, d
    assert abs(mix.kinetic_energy() / f64.kinetic_energy() - 1) < 1e-7
    assert mix.status() == 0


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_precision_config_p5_500_steps(flux):
    """The precision configuration (64^3, p = 5, 500 RK4 steps at CFL 0.1) on a
    16^3 mesh of the same box: the mixed path stays within 1e-6 of FP64 per
    variable after 500 steps, and both L2 errors against the exact advected
    vortex agree to that difference."""
    mesh = dg_b200.periodic_box((16, 16, 16), (0, 0, 0), (10.0, 10.0, 10.0))
    f64 = dg_b200.Case(mesh, 5, flux=flux, gas_constant=1.0, precision="fp64")
    mix = dg_b200.Case(mesh, 5, flux=flux, gas_constant=1.0, precision="mixed_fp32")
    U0 = f64.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = f64.cfl_time_step(U0, 0.1)
    mix.set_state(U0)
    f64.rk4(dt, 500)
    mix.rk4(dt, 500)
    d = rel_l2(mix.get_state(), f64.get_state())
    assert d.max() < TOL, d
    t = 500 * dt
    e64 = f64.l2_error("IsentropicVortexXY", VORTEX_XY, t)
    emx = mix.l2_error("IsentropicVortexXY", VORTEX_XY, t)
    print(f"p=5 16^3 500 steps {flux}: mixed vs FP64 {d}, L2 error FP64 {e64}, mixed {emx}")
    # at p = 5 the discretisation error (~5e-7 in rho) is as small as the FP32
    # residual's rounding, so the two errors against the exact vortex differ by
    # at most the distance between the solutions (triangle inequality; the
    # states are O(1), rho E ~ 3)
    assert np.all(np.abs(emx - e64) <= 3.0 * TOL), (emx, e64)
    assert mix.status() == 0 and f64.status() == 0


def _tc_variant(case):
    vs = case.stage_variants()
    tc = [i for i, v in enumerate(vs) if "tc" in v[4].split("+")]
    assert tc, "p = 3 compiles a tensor-core variant"
    return tc[0]


@pytest.mark.parametrize("n", [(7, 1, 1), (5, 3, 2), (3, 2, 3)])
def test_tensor_core_residual_and_modes_match_fp64(n):
    """The tensor-core kernel (split-BF16 volume GEMMs on tcgen05) on meshes whose
    element count leaves a partial tile (7 = 6 + 1) or none, rotated elements:
    residual, inverse-mass residual and RK4 steps against the FP64 path at the
    FP32 residual's accuracy."""
    mesh = dg_b200.periodic_box(n, (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=13)
    f64 = dg_b200.Case(mesh, 3, gas_constant=1.0, precision="fp64")
    tc = dg_b200.Case(mesh, 3, gas_constant=1.0, precision="mixed_fp32")
    f32 = dg_b200.Case(mesh, 3, gas_constant=1.0, precision="mixed_fp32")  # the CUDA-core FP32 residual
    tc.stage_variant = _tc_variant(tc)
    U = f64.project_ic("IsentropicVortexXY", VORTEX_XY)
    tc.set_state(U)
    f32.set_state(U)
    R64, Rtc, R32 = f64.residual(), tc.residual(), f32.residual()
    scale = np.abs(R64).max()
    assert np.abs(Rtc - R64).max() < 1e-5 * scale
    dt = f64.cfl_time_step(U, 0.1)
    M64, Mtc, M32 = f64.mass_inverse_residual(dt), tc.mass_inverse_residual(dt), f32.mass_inverse_residual(dt)
    # the inverse mass amplifies FP32 rounding alike on both FP32 residuals
    etc, e32 = np.abs(Mtc - M64).max(), np.abs(M32 - M64).max()
    assert etc < 1e-4 * np.abs(M64).max() and etc < 4 * e32, (etc, e32)
    f64.rk4(dt, 10)
    tc.rk4(dt, 10)
    assert rel_l2(tc.get_state(), f64.get_state()).max() < TOL
    assert tc.status() == 0


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_tensor_core_stepping_within_bound(flux):
    """60 RK4 steps of the 8^3 p = 3 vortex and 40 of low-Mach Taylor-Green on the
    tensor-core kernel: within 1e-6 of FP64 per variable."""
    mesh = dg_b200.periodic_box((8, 8, 8), (0, 0, 0), (10.0, 10.0, 10.0), rotate_seed=3)
    f64 = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0, precision="fp64")
    tc = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0, precision="mixed_fp32")
    tc.stage_variant = _tc_variant(tc)
    U0 = f64.project_ic("IsentropicVortexXY", VORTEX_XY)
    dt = f64.cfl_time_step(U0, 0.1)
    tc.set_state(U0)
    f64.rk4(dt, 60)
    tc.rk4(dt, 60)
    d = rel_l2(tc.get_state(), f64.get_state())
    print(f"tensor-core 8^3 p=3 vortex 60 steps {flux}: {d}")
    assert d.max() < TOL, d
    L = 2 * np.pi
    mesh = dg_b200.periodic_box((8, 8, 8), (0, 0, 0), (L, L, L))
    f64 = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0, precision="fp64")
    tc = dg_b200.Case(mesh, 3, flux=flux, gas_constant=1.0, precision="mixed_fp32")
    tc.stage_variant = _tc_variant(tc)
    U0 = f64.project_ic("TaylorGreen", [0.1])
    dt = f64.cfl_time_step(U0, 0.1)
    tc.set_state(U0)
    f64.rk4(dt, 40)
    tc.rk4(dt, 40)
    d = rel_l2(tc.get_state(), f64.get_state())
    print(f"tensor-core 8^3 p=3 Taylor-Green M=0.1 40 steps {flux}: {d}")
    assert d.max() < TOL, d
    assert tc.status() == 0
