"""Pins the CPU oracle to the reference's own golden vectors (CPU only).

The oracle restates IhmeGroup/DG-MPI's dense algorithm; these tests check it
against every number the reference publishes for this path: the 3D vortex
regression errors, its Gauss-Legendre tables, the basis / node unit tests,
and the flux properties of its (disabled) physics tests.
"""
import numpy as np
import pytest

import dg_b200
import pyoracle


def test_gauss_legendre_matches_reference_tables(golden):
    # reference tables: src/numerics/nodes.cpp, src/numerics/quadrature/segment.cpp
    worst = 0.0
    for order, tab in golden["gauss_legendre"]["by_order"].items():
        x, w = pyoracle.gauss_legendre(int(order))
        xr, wr = np.array(tab["nodes"]), np.array(tab["weights"])
        assert x.shape == xr.shape
        worst = max(worst, np.abs(x - xr).max(), np.abs(w - wr).max())
    assert worst <= 4.5e-16  # within an ulp or two of the 32-digit tables


@pytest.mark.parametrize("order", range(1, 20))
def test_quadrature_weights_sum_to_measure(order, golden):
    # test/numerics/quadrature/test_quadrature.cpp:19-122 (segment, quad, hex)
    tol = golden["tolerance"]["double"]
    lib = pyoracle.library()
    x, w = pyoracle.gauss_legendre(lib.orc_segment_quadrature_order(order))
    assert abs(w.sum() - 2.0) < tol
    xq, wq = pyoracle.gauss_legendre(lib.orc_quad_quadrature_order(order))
    assert abs(np.outer(wq, wq).sum() - 4.0) < tol
    xh, wh = pyoracle.gauss_legendre(lib.orc_hex_quadrature_order(order))
    assert abs(np.einsum("i,j,k->ijk", wh, wh, wh).sum() - 8.0) < tol


def test_equidistant_nodes(golden):
    lib = pyoracle.library()
    for start, stop, n, expected in golden["equidistant_nodes"]["cases"]:
        x = np.zeros(max(n, 1))
        lib.orc_equidistant_nodes(start, stop, n, pyoracle._d(x))
        np.testing.assert_allclose(x, expected, atol=1e-13)


@pytest.mark.parametrize("p", range(1, 6))
def test_lagrange_hex_is_nodal(p):
    # test/numerics/basis/test_basis.cpp:217-262
    n = p + 1
    xn = np.linspace(-1, 1, n)
    pts = np.array([[xn[i], xn[j], xn[k]] for k in range(n) for j in range(n) for i in range(n)])
    val = np.zeros((n ** 3, n ** 3))
    pyoracle.library().orc_lagrange_hex_val(p, n ** 3, pyoracle._d(np.ascontiguousarray(pts)), pyoracle._d(val))
    np.testing.assert_allclose(val, np.eye(n ** 3), atol=1e-13)


def test_lagrange_hex_p1_gradient(golden):
    gold = golden["lagrange_hex_p1_grad_at_minus1"]
    grad = np.zeros((1, 8, 3))
    pts = np.array([gold["xi"]], np.float64)
    pyoracle.library().orc_lagrange_hex_grad(1, 1, pyoracle._d(pts), pyoracle._d(grad))
    np.testing.assert_allclose(grad[0], gold["grad"], atol=1e-13)


def _random_state(rng, n=1):
    rho = rng.uniform(0.5, 2.0, n)
    u = rng.uniform(-1, 1, (n, 3))
    p = rng.uniform(0.5, 2.0, n)
    E = p / 0.4 + 0.5 * rho * (u ** 2).sum(1)
    return np.column_stack([rho, rho * u[:, 0], rho * u[:, 1], rho * u[:, 2], E])


@pytest.mark.parametrize("kind", ["LaxFriedrichs", "HLLC"])
def test_numerical_flux_consistency_and_conservation(kind):
    # properties of the reference's test_physics.cpp:479-576, restated in 3D:
    # F(U, U, N) = F(U) . N and F(UL, UR, N) = -F(UR, UL, -N)
    rng = np.random.default_rng(7)
    for _ in range(50):
        UL, UR = _random_state(rng, 2)
        N = rng.normal(size=3)
        F, rc = pyoracle.num_flux(kind, 1.4, UL, UL, N)
        assert rc == 0
        Fd = pyoracle.conv_flux(1.4, UL).reshape(3, 5)
        np.testing.assert_allclose(F, Fd.T @ N, rtol=1e-12, atol=1e-12)
        F1, _ = pyoracle.num_flux(kind, 1.4, UL, UR, N)
        F2, _ = pyoracle.num_flux(kind, 1.4, UR, UL, -N)
        np.testing.assert_allclose(F1, -F2, rtol=1e-12, atol=1e-12)


def test_face_orientation_orders_are_permutations():
    for n1 in range(1, 9):
        orders = [tuple(pyoracle.face_pts_order(o, n1 * n1)) for o in range(8)]
        for o in orders:
            assert sorted(o) == list(range(n1 * n1))
        if n1 >= 2:
            assert len(set(orders)) == 8  # the dihedral group acts faithfully


@pytest.mark.slow
def test_vortex3d_regression_known_answer(golden):
    """examples/euler/3D/isentropic_vortex/regression_data.txt: p=3, 4^3 periodic
    [0,1]^3, HLLC, RK4 dt=1e-3 to t=1 (1000 steps); L2 errors vs the IC."""
    g = golden["vortex3d_regression"]
    mesh = dg_b200.periodic_box((4, 4, 4), (0, 0, 0), (1, 1, 1))
    oc = pyoracle.OracleCase.from_mesh(mesh, g["order"], flux=g["flux"], gamma=g["gamma"],
                                       gas_constant=g["gas_constant"])
    U = oc.project_ic("IsentropicVortex")
    nsteps = int(g["end"] / g["timestep"])  # base.cpp:383 truncation: 1000
    U = oc.rk4(U, g["timestep"], nsteps)
    err = oc.l2_error(U, "IsentropicVortex")
    ref = np.array(g["l2_errors"])
    assert oc.flux_failures() == 0
    # rho, rho u, rho w, rho E to 1e-12 relative; rho v is rounding noise (~1e-15)
    for s in (0, 1, 3, 4):
        assert abs(err[s] - ref[s]) <= 1e-12 * ref[s], (s, err[s], ref[s])
    assert err[2] < 1e-13 and ref[2] < 1e-13


def test_rotated_mesh_gives_same_physics():
    """A mesh whose elements use rotated local numberings (non-trivial face
    orientations) advances the same physical solution (p=2, 3^3, 5 steps)."""
    ref = dg_b200.periodic_box((3, 3, 3), (0, 0, 0), (1, 1, 1))
    rot = dg_b200.periodic_box((3, 3, 3), (0, 0, 0), (1, 1, 1), rotate_seed=12345)
    assert not np.array_equal(ref.elem_to_node_ids, rot.elem_to_node_ids)
    errs = []
    for mesh in (ref, rot):
        oc = pyoracle.OracleCase.from_mesh(mesh, 2, flux="LaxFriedrichs", gas_constant=1.0)
        U = oc.project_ic("IsentropicVortex")
        U = oc.rk4(U, 2e-3, 5)
        errs.append(oc.l2_error(U, "IsentropicVortex"))
    np.testing.assert_allclose(errs[0][[0, 1, 3, 4]], errs[1][[0, 1, 3, 4]], rtol=1e-10)


def test_oracle_conserves_on_periodic_mesh():
    # sum over elements of the cell integral of R is zero on a periodic mesh:
    # integral of phi_b summed with the constant function -> mass of R
    mesh = dg_b200.periodic_box((3, 2, 2), (0, 0, 0), (1, 1, 1), rotate_seed=3)
    oc = pyoracle.OracleCase.from_mesh(mesh, 2, flux="HLLC", gas_constant=1.0)
    U = oc.project_ic("IsentropicVortex")
    R = oc.residual(U)
    # a Lagrange basis sums to one, so sum_b R[e, b, s] is the test with phi = 1
    total = R.sum(axis=(0, 1))
    # scale by the largest variable: rho v is identically zero up to rounding here
    assert np.all(np.abs(total) < 1e-12 * np.abs(R).sum(axis=(0, 1)).max())
