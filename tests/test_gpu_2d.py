"""The 2D quadrilateral path on the GPU (dg2d_*, csrc/dg_2d.cu) against the
2D oracle (the reference's dense Solver<2> algorithm) and against the
reference's 2D convergence table.

Bars as for the 3D FP64 path: one residual <= 1e-11 relative L2 per variable,
time stepping <= 1e-12, projection <= 1e-13; the convergence-table entries to
the oracle's pin, 2e-6 relative (see test_oracle2d.py).
"""
import os

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401
import dg_b200
import pyoracle
from test_oracle2d import TABLE, VORTEX, PIN_RTOL

pytestmark = pytest.mark.gpu

XY = [1.0, 0.4, -0.3, 1.0, 5.0, 0.7, -0.2, 10.0, 9.0]  # x-y vortex, periodic on the box below


def rel_l2(a, b):
    a = np.asarray(a).reshape(-1, a.shape[-1])
    b = np.asarray(b).reshape(-1, b.shape[-1])
    return np.linalg.norm(a - b, axis=0) / np.maximum(np.linalg.norm(b, axis=0), 1e-300)


def _pair(p, flux, n=(4, 3), seed=5):
    m = dg_b200.periodic_box_2d(n, (-5.0, -4.5), (10.0, 9.0), rotate_seed=seed)
    gpu = dg_b200.Case2D(m, p, flux=flux, gas_constant=1.0)
    orc = pyoracle.OracleCase2D.from_mesh(m, p, flux=flux, gas_constant=1.0)
    return m, gpu, orc


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
@pytest.mark.parametrize("p", [0, 1, 2, 3, 4, 5])
def test_residual_matches_oracle_2d(p, flux):
    _, gpu, orc = _pair(p, flux)
    U = orc.project_ic("IsentropicVortexXY", XY)
    gpu.set_state(U)
    d = rel_l2(gpu.residual(), orc.residual(U))
    assert d.max() < 1e-11, d
    assert gpu.status() == 0


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
@pytest.mark.parametrize("p", [1, 3, 5])
def test_rk4_and_fe_steps_match_oracle_2d(p, flux):
    _, gpu, orc = _pair(p, flux)
    U = orc.project_ic("IsentropicVortexXY", XY)
    gpu.set_state(U)
    gpu.rk4(2e-3, 10)
    assert rel_l2(gpu.get_state(), orc.rk4(U, 2e-3, 10)).max() < 1e-12
    gpu.set_state(U)
    gpu.fe(1e-3, 3)
    assert rel_l2(gpu.get_state(), orc.fe(U, 1e-3, 3)).max() < 1e-12
    gpu.rk4(1e-3, 2)  # the RK4 graph after an odd number of FE steps (buffers swapped)
    assert rel_l2(gpu.get_state(), orc.rk4(orc.fe(U, 1e-3, 3), 1e-3, 2)).max() < 1e-12


@pytest.mark.parametrize("p", [0, 1, 2, 3, 4, 5])
def test_projection_and_error_match_oracle_2d(p):
    _, gpu, orc = _pair(p, "HLLC")
    Ug = gpu.project_ic("IsentropicVortex", VORTEX)
    Uo = orc.project_ic("IsentropicVortex", VORTEX)
    assert rel_l2(Ug, Uo).max() < 1e-13
    Uo2 = orc.rk4(Uo, 1e-3, 5)
    gpu.set_state(Uo2)
    np.testing.assert_allclose(gpu.l2_error("IsentropicVortex", VORTEX, 5e-3),
                               orc.l2_error(Uo2, "IsentropicVortex", VORTEX, 5e-3), rtol=1e-10)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_reference_convergence_table_on_gpu(p):
    """The reference's 2D convergence table (N = 2, 4, 8, 16) reproduced by
    the GPU path to the oracle's pin, and the error falling at order p+1
    from N = 16 to 32."""
    errs = []
    for k, N in enumerate([2, 4, 8, 16, 32]):
        m = dg_b200.periodic_box_2d((N, N), (-5.0, -5.0), (10.0, 10.0))
        gpu = dg_b200.Case2D(m, p, flux="HLLC", gas_constant=1.0)
        gpu.project_ic("IsentropicVortex", VORTEX)
        gpu.rk4(1e-3, 1000)
        e = gpu.l2_error("IsentropicVortex", VORTEX, 1.0)[0]
        errs.append(e)
        if k < 4:
            assert abs(e / TABLE[p][k] - 1.0) < PIN_RTOL, (N, e, TABLE[p][k])
        assert gpu.status() == 0
    rate = np.log(errs[3] / errs[4]) / np.log(2.0)
    assert rate > p + 0.5, (rate, errs)


def test_reference_quad_1x1_mesh_on_gpu():
    m = dg_b200.read_mesh_h5(os.path.join(os.path.dirname(__file__), "golden", "meshes", "quad_1x1.h5"))
    gpu = dg_b200.Case2D(m, 3, flux="HLLC", gas_constant=1.0)
    U = gpu.project_ic("Uniform", [1.2, 0.3, -0.4, 2.5])
    assert np.abs(gpu.residual()).max() < 1e-13
    gpu.rk4(1e-3, 20)
    assert np.abs(gpu.get_state() - U).max() < 1e-13


def test_nonphysical_state_is_reported_2d():
    _, gpu, orc = _pair(2, "HLLC")
    U = orc.project_ic("IsentropicVortexXY", XY)
    U[1, :, 0] = -1.0
    gpu.set_state(U)
    with pytest.raises(dg_b200.DGError, match="NONPHYSICAL"):
        gpu.rk4(1e-3, 1)


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_reference_quad_2x2_mesh_with_boundary_edges(flux):
    """The reference's non-periodic 2x2 example mesh (its boundary edges carry
    no interior face): the residual adds nothing on those edges, as the
    reference's residual loops over the interior faces only; GPU against the
    oracle on a vortex state, and FE steps."""
    m = dg_b200.read_mesh_h5(os.path.join(os.path.dirname(__file__), "golden", "meshes", "quad_2x2.h5"))
    assert m.interior_faces.shape[0] == 4 and m.elem_to_node_ids.shape[0] == 4
    gpu = dg_b200.Case2D(m, 2, flux=flux, gas_constant=1.0)
    orc = pyoracle.OracleCase2D.from_mesh(m, 2, flux=flux, gas_constant=1.0)
    data = [1.0, 0.3, 0.2, 1.0, 5.0, 0.4, 0.6, 1e30, 1e30]
    U = orc.project_ic("IsentropicVortexXY", data)
    assert rel_l2(gpu.project_ic("IsentropicVortexXY", data), U).max() < 1e-13
    assert rel_l2(gpu.residual(), orc.residual(U)).max() < 1e-11
    gpu.fe(1e-3, 2)
    assert rel_l2(gpu.get_state(), orc.fe(U, 1e-3, 2)).max() < 1e-12
