"""The 2D oracle (oracle/oracle2d.c: Solver<2> with LagrangeQuad, the dense
per-element algorithm) against the reference's 2D convergence table, and its
properties; the 2D mesh generator and boundary checks of the 2D C ABI that
need no GPU.

Pin: examples/isentropic_vortex/convergence.py of the reference lists the
density L2 error of the 2D isentropic vortex (input.toml there: HLLC,
LagrangeQuad, RK4, dt = 1e-3 to t = 1, gamma 1.4, GasConstant 1, data
[1, 1, 1, 1, 5]) on N x N boxes for p = 1, 2, 3.  The meshes
(meshes/box_NxN.h5) are not in the reference; periodic boxes on [-5, 5]^2
reproduce the table to within 1.1e-6 relative for every entry checked here
(N = 2 .. 16), while the closest alternative scheme -- p+2 Gauss points per
edge instead of the segment rule's p+1 -- is off by 3e-4 to 3e-2.  The
remaining ~1e-7 is not explained (the table comes from GPU runs of the
reference; a float32 time step does not account for it), so the pin is a
relative 2e-6, not the digits.
"""
import os

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401  (puts the package and the oracle on sys.path)
import dg_b200
import pyoracle

TABLE = {  # examples/isentropic_vortex/convergence.py:51-86, N = 2, 4, 8, 16
    1: [4.057487237640151206408e-02, 3.659091741930729779764e-02, 1.399040502291195101070e-02,
        3.736915003326653998000e-03],
    2: [3.932754850914681188367e-02, 1.414430149472130186783e-02, 3.248199949411992391163e-03,
        3.915751398100587301818e-04],
    3: [2.911726700453628677301e-02, 6.747203591607888774340e-03, 5.564165617240108456867e-04,
        3.771907882313834693960e-05],
}
VORTEX = [1.0, 1.0, 1.0, 1.0, 5.0]
PIN_RTOL = 2e-6
QUAD_FACE_NODES = [(0, 1), (1, 3), (3, 2), (2, 0)]


def _run(N, p, flux="HLLC", steps=1000, rotate=0):
    m = dg_b200.periodic_box_2d((N, N), (-5.0, -5.0), (10.0, 10.0), rotate_seed=rotate)
    orc = pyoracle.OracleCase2D.from_mesh(m, p, flux=flux, gas_constant=1.0)
    U = orc.project_ic("IsentropicVortex", VORTEX)
    U = orc.rk4(U, 1e-3, steps)
    return orc, U, orc.l2_error(U, "IsentropicVortex", VORTEX, steps * 1e-3)


@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("k,N", [(0, 2), (1, 4), (2, 8)])
def test_oracle2d_reproduces_reference_convergence_table(p, k, N):
    _, _, err = _run(N, p)
    assert abs(err[0] / TABLE[p][k] - 1.0) < PIN_RTOL, (err[0], TABLE[p][k])


def test_oracle2d_is_invariant_under_element_rotations():
    _, _, e0 = _run(4, 2, steps=50)
    _, _, e1 = _run(4, 2, steps=50, rotate=7)
    np.testing.assert_allclose(e1, e0, rtol=1e-12)


@pytest.mark.parametrize("flux", ["LaxFriedrichs", "HLLC"])
def test_oracle2d_residual_conserves(flux):
    """Sum of the residual over all basis functions (they add up to one) is
    the integral of a divergence over a periodic domain: zero."""
    m = dg_b200.periodic_box_2d((3, 5), (-5.0, -4.0), (10.0, 9.0), rotate_seed=3)
    orc = pyoracle.OracleCase2D.from_mesh(m, 3, flux=flux, gas_constant=1.0)
    U = orc.project_ic("IsentropicVortexXY", [1, 0.3, -0.2, 1, 5, 0.5, 0.5, 10, 9])
    R = orc.residual(U)
    total = R.sum(axis=(0, 1))
    assert np.all(np.abs(total) < 1e-12 * np.abs(R).sum(axis=(0, 1)).max()), total
    assert orc.flux_failures() == 0


def test_reference_quad_1x1_mesh_keeps_a_uniform_state():
    """The reference's periodic one-element mesh file through the library's
    reader and the oracle: a uniform state has a zero residual."""
    m = dg_b200.read_mesh_h5(os.path.join(os.path.dirname(__file__), "golden", "meshes", "quad_1x1.h5"))
    orc = pyoracle.OracleCase2D.from_mesh(m, 2, flux="HLLC", gas_constant=1.0)
    U = orc.project_ic("Uniform", [1.2, 0.3, -0.4, 2.5])
    R = orc.residual(U)
    assert np.abs(R).max() < 1e-13
    np.testing.assert_allclose(U[0, :, 0], 1.2, rtol=1e-14)


@pytest.mark.parametrize("seed", [0, 11])
def test_periodic_box_2d_faces_match_geometrically(seed):
    m = dg_b200.periodic_box_2d((4, 3), (-1.0, 2.0), (3.0, 2.0), rotate_seed=seed)
    assert (m.dim, m.elem_to_node_ids.shape, m.interior_faces.shape) == (2, (12, 4), (24, 8))
    x = m.node_coords
    ext = np.array([3.0, 2.0])
    seen = set()
    for row in m.interior_faces:
        assert row[3] == 0 and row[7] == 1
        pL = x[m.elem_to_node_ids[row[1]][list(QUAD_FACE_NODES[row[2]])]]
        pR = x[m.elem_to_node_ids[row[5]][list(QUAD_FACE_NODES[row[6]])]]
        k = np.round((pL.mean(0) - pR.mean(0)) / ext)
        # the two sides traverse the shared edge in opposite directions
        np.testing.assert_allclose(pL - k * ext, pR[::-1], atol=1e-14)
        seen |= {(row[1], row[2]), (row[5], row[6])}
    assert len(seen) == 48
    # positive Jacobians: local node 1 - 0 and 2 - 0 span a positive area
    for e in m.elem_to_node_ids:
        a, b = x[e[1]] - x[e[0]], x[e[2]] - x[e[0]]
        assert a[0] * b[1] - a[1] * b[0] > 0


def test_2d_context_refuses_non_parallelograms_and_3d_meshes():
    m = dg_b200.periodic_box_2d((2, 2), (0.0, 0.0), (1.0, 1.0))
    m.node_coords[4] += [0.1, 0.05]  # the shared centre node: four non-parallelograms
    with pytest.raises(dg_b200.DGError, match="not a parallelogram"):
        dg_b200.Case2D(m, 2)
    with pytest.raises(ValueError, match="quadrilateral meshes"):
        dg_b200.Case2D(dg_b200.periodic_box((2, 2, 2)), 2)
    with pytest.raises(dg_b200.DGError, match="FP64"):
        lib = dg_b200.library()
        import ctypes
        keep = []
        md = dg_b200._mesh2d_desc(dg_b200.periodic_box_2d((2, 2)), keep)
        cd = dg_b200._CaseDesc(1, 0, 1.4, 1.0, 1, 0)
        h = ctypes.c_void_p()
        rc = lib.dg2d_create(ctypes.byref(cd), ctypes.byref(md), ctypes.byref(h))
        raise dg_b200.DGError(rc, lib.dg_last_error(None).decode())
