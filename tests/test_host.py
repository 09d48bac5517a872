"""Host side of the drop-in (CPU only): the C ABI library loads and exports
every declared symbol, the product's own tables agree with the oracle's
restatement of the reference, the periodic mesh generator produces the
reference's mesh semantics, and mesh validation rejects what the device path
cannot handle -- all without touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import dg_b200
import pyoracle
from conftest import ROOT, gpu_available


def declared_symbols():
    with open(os.path.join(ROOT, "include", "dg_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(dg_b200.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    lib = dg_b200.library()
    for n in declared_symbols():
        assert getattr(lib, n).argtypes is not None, n


def test_bounded_wait_probe_rejects_limits_out_of_range():
    """dg_probe_bounded_wait checks its limit before any device work."""
    lib = dg_b200.library()
    for limit in (-1, 4_000_000_001):
        assert lib.dg_probe_bounded_wait(0, limit, 0, None) == 1  # DG_ERR_ARG
        assert b"limit" in lib.dg_last_error(None)


@pytest.mark.parametrize("n", range(1, 13))
def test_gauss_legendre_matches_oracle(n):
    x, w = dg_b200.gauss_legendre(n)
    xo, wo = pyoracle.gauss_legendre(2 * n - 1)
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_array_equal(w, wo)


@pytest.mark.parametrize("n1", range(1, 9))
def test_face_orientation_orders_match_reference_walks(n1):
    # product: closed-form dihedral maps; oracle: shape.cpp:326-428 walks
    for o in range(8):
        np.testing.assert_array_equal(dg_b200.face_orientation_order(o, n1 * n1),
                                      pyoracle.face_pts_order(o, n1 * n1))


@pytest.mark.parametrize("p", range(0, 6))
def test_1d_tables_reproduce_reference_3d_tables(p):
    """The kernels' 1D tables, tensorised, equal the reference's dense 3D
    basis / gradient tables at the volume points (helpers.cpp:143-183)."""
    B, D, Mi = dg_b200.basis_tables(p)
    lib = pyoracle.library()
    m = p + 2
    x, _ = pyoracle.gauss_legendre(lib.orc_hex_quadrature_order(p))
    assert x.size == m
    pts = np.array([[x[i], x[j], x[k]] for k in range(m) for j in range(m) for i in range(m)])
    nb = (p + 1) ** 3
    val = np.zeros((m ** 3, nb))
    grad = np.zeros((m ** 3, nb, 3))
    lib.orc_lagrange_hex_val(p, m ** 3, pyoracle._d(np.ascontiguousarray(pts)), pyoracle._d(val))
    lib.orc_lagrange_hex_grad(p, m ** 3, pyoracle._d(np.ascontiguousarray(pts)), pyoracle._d(grad))
    B3 = np.einsum("kc,jb,ia->kjicba", B, B, B).reshape(m ** 3, nb)
    np.testing.assert_allclose(B3, val, atol=1e-14)
    if p > 0:
        Gx = np.einsum("kc,jb,ia->kjicba", B, B, D).reshape(m ** 3, nb)
        Gz = np.einsum("kc,jb,ia->kjicba", D, B, B).reshape(m ** 3, nb)
        np.testing.assert_allclose(Gx, grad[:, :, 0], atol=1e-13)
        np.testing.assert_allclose(Gz, grad[:, :, 2], atol=1e-13)
    # Minv is the inverse of the exactly integrated 1D mass matrix
    n = p + 1
    xm, wm = np.polynomial.legendre.leggauss(2 * p + 2)
    xn = np.linspace(-1, 1, n) if n > 1 else np.zeros(1)
    phi = np.ones((xm.size, n))
    for i in range(n):
        for j in range(n):
            if i != j:
                phi[:, i] *= (xm - xn[j]) / (xn[i] - xn[j])
    M = (phi * wm[:, None]).T @ phi
    np.testing.assert_allclose(Mi @ M, np.eye(n), atol=1e-11)


@pytest.mark.parametrize("seed", [0, 1, 99])
@pytest.mark.parametrize("p", [1, 3])
def test_mesh_generator_matches_reference_face_semantics(seed, p):
    """For every interior face, the left face point quad_idx_L[q] and the
    right face point quad_idx_R[q] coincide physically (modulo the period),
    and the normal (computed the reference's way, from the left element)
    points out of the left element with |N| = face area / 4."""
    L = np.array([1.0, 2.0, 0.5])
    mesh = dg_b200.periodic_box((3, 2, 4), (0.1, -0.2, 0.0), L, rotate_seed=seed)
    oc = pyoracle.OracleCase.from_mesh(mesh, p, gas_constant=1.0)
    iL, iR = oc.quad_idx()
    N = oc.face_normals()
    ifd = mesh.iface_data()
    h = L / np.array([3, 2, 4])
    centers = mesh.node_coords[mesh.elem_to_node_ids].mean(axis=1)
    for f in range(ifd.shape[0]):
        eL, fL, _, eR, fR, _ = ifd[f]
        XL = oc.face_points(eL, fL)[iL[f]]
        XR = oc.face_points(eR, fR)[iR[f]]
        d = XL - XR
        d -= L * np.round(d / L)
        assert np.abs(d).max() < 1e-12
        n = N[f, 0]
        out = XL[0] - centers[eL]
        assert np.dot(n, out) > 0
        axis = int(np.argmax(np.abs(n)))
        area = np.prod(np.delete(h, axis))
        assert abs(np.linalg.norm(n) - area / 4) < 1e-12
        assert np.allclose(N[f], N[f, 0], atol=1e-14)


def test_mesh_validation_rejects_boundary_faces_before_touching_the_gpu():
    mesh = dg_b200.periodic_box((2, 2, 2))
    broken = dg_b200.Mesh(mesh.node_coords, mesh.elem_to_node_ids, mesh.interior_faces[:-1].copy())
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.Case(broken, 1)
    assert ei.value.code == 5 and "boundary face" in str(ei.value)


def test_non_affine_elements_pass_validation_and_folded_ones_do_not():
    """Bent (trilinear) elements are accepted -- without a GPU creation then stops
    at the device -- while an element with a non-positive Jacobian somewhere is
    rejected on the host, as are non-affine cases in a batch."""
    from conftest import gpu_available
    mesh = dg_b200.periodic_box((2, 2, 2))
    coords = mesh.node_coords.copy()
    coords[13] += [0.05, 0.0, 0.0]  # the centre node: every element around it bends
    bent = dg_b200.Mesh(coords, mesh.elem_to_node_ids, mesh.interior_faces)
    if not gpu_available():
        with pytest.raises(dg_b200.DGError, match="DG_ERR_CUDA"):
            dg_b200.Case(bent, 2)
    folded = mesh.node_coords.copy()
    folded[13] += [0.9, 0.0, 0.0]  # past the neighbouring nodes: elements fold
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.Case(dg_b200.Mesh(folded, mesh.elem_to_node_ids, mesh.interior_faces), 2)
    assert ei.value.code == 1 and "non-positive Jacobian" in str(ei.value)
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.Batch([(mesh, 2), (bent, 2)])
    assert ei.value.code == 5 and "non-affine" in str(ei.value)


def test_mesh_validation_rejects_out_of_range_entries():
    mesh = dg_b200.periodic_box((2, 2, 2))
    faces = mesh.interior_faces.copy()
    faces[0, 3] = 9  # orientation must be 0..7
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.Case(dg_b200.Mesh(mesh.node_coords, mesh.elem_to_node_ids, faces), 1)
    assert ei.value.code == 1


def test_unsupported_order_and_precision():
    mesh = dg_b200.periodic_box((2, 2, 2))
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.Case(mesh, 6)
    assert ei.value.code == 5


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_cleanly():
    mesh = dg_b200.periodic_box((2, 2, 2))
    with pytest.raises(dg_b200.DGError) as ei:
        dg_b200.Case(mesh, 1)
    assert ei.value.code == 2


FUZZ_CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import dg_b200
rng = np.random.default_rng(int(sys.argv[2]))
mesh = dg_b200.periodic_box((2, 3, 2), rotate_seed=3)
codes = {}
for it in range(int(sys.argv[3])):
    faces = mesh.interior_faces.copy()
    e2n = mesh.elem_to_node_ids.copy()
    coords = mesh.node_coords.copy()
    for _ in range(int(rng.integers(1, 4))):
        kind = int(rng.integers(0, 3))
        if kind == 0:
            i, j = int(rng.integers(0, faces.shape[0])), int(rng.integers(0, 8))
            faces[i, j] = int(rng.choice([0, 1, 5, 7, 8, 23, 2**31 - 1, 2**32 - 1]))
        elif kind == 1:
            i, j = int(rng.integers(0, e2n.shape[0])), int(rng.integers(0, 8))
            e2n[i, j] = int(rng.choice([0, coords.shape[0] - 1, coords.shape[0], 2**32 - 1]))
        else:
            coords[int(rng.integers(0, coords.shape[0])), int(rng.integers(0, 3))] = float(
                rng.choice([np.nan, np.inf, -1e300, 0.0]))
    try:
        c = dg_b200.Case(dg_b200.Mesh(coords, e2n, faces), int(rng.integers(0, 4)))
        c.close()
        codes[0] = codes.get(0, 0) + 1
    except dg_b200.DGError as e:
        codes[e.code] = codes.get(e.code, 0) + 1
# the halo plan of a slab partition and the 2D context take the same tables
pm, part = dg_b200.partition_periodic_box((2, 2, 4), (0, 0, 0), (1, 1, 1), 2, 0)
m2 = dg_b200.periodic_box_2d((3, 2), rotate_seed=4)
for it in range(int(sys.argv[3])):
    faces = pm.interior_faces.copy()
    i, j = int(rng.integers(0, faces.shape[0])), int(rng.choice([1, 2, 5, 6]))
    faces[i, j] = int(rng.choice([5, 6, 2**31 - 1, 2**32 - 1]))
    try:
        dg_b200.halo_plan(dg_b200.Mesh(pm.node_coords, pm.elem_to_node_ids, faces), part)
        codes[0] = codes.get(0, 0) + 1
    except dg_b200.DGError as e:
        codes[e.code] = codes.get(e.code, 0) + 1
    faces2, e2n2 = m2.interior_faces.copy(), m2.elem_to_node_ids.copy()
    if rng.integers(0, 2):
        faces2[int(rng.integers(0, faces2.shape[0])), int(rng.integers(0, 8))] = int(rng.choice([2, 4, 2**32 - 1]))
    else:
        e2n2[int(rng.integers(0, e2n2.shape[0])), int(rng.integers(0, 4))] = int(rng.choice([12, 2**32 - 1]))
    try:
        c = dg_b200.Case2D(dg_b200.Mesh(m2.node_coords, e2n2, faces2), 1)
        c.close()
        codes[0] = codes.get(0, 0) + 1
    except dg_b200.DGError as e:
        codes[e.code] = codes.get(e.code, 0) + 1
    # a batch with one corrupt case among valid ones
    bad = dg_b200.Mesh(mesh.node_coords, mesh.elem_to_node_ids, mesh.interior_faces.copy())
    bad.interior_faces[int(rng.integers(0, bad.interior_faces.shape[0])), int(rng.choice([1, 5]))] = 2**32 - 1
    try:
        b = dg_b200.Batch([(mesh, 2), (bad, 3)])
        b.close()
        codes[0] = codes.get(0, 0) + 1
    except dg_b200.DGError as e:
        codes[e.code] = codes.get(e.code, 0) + 1
print(sorted(codes.items()))
"""


def test_corrupt_mesh_tables_fail_cleanly(tmp_path):
    """Random corruptions of the face table (element, face, orientation and
    rank entries, negative values included, which the unsigned table holds
    as huge ones), the element-to-node table and the node coordinates (NaN,
    infinities) end in an error code from the host-side validation (or, where
    the corruption leaves a valid mesh, in a context or the no-GPU error),
    never in a crash -- for 3D contexts, the halo plan of a partition, 2D
    contexts and batches; run in a child process so that a fault would fail
    this test."""
    import subprocess
    import sys
    script = tmp_path / "fuzz.py"
    script.write_text(FUZZ_CHILD)
    r = subprocess.run([sys.executable, str(script), os.path.join(ROOT, "dg-mpi_b200"), "11", "300"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    counts = dict(eval(r.stdout.strip()))
    assert set(counts) <= {0, 1, 2, 5}, counts
    assert counts.get(1, 0) + counts.get(5, 0) > 400, counts


NULL_CHILD = r"""
import ctypes, re, sys
sys.path.insert(0, sys.argv[1])
import dg_b200
lib = dg_b200.library()
text = re.sub(r"/\*.*?\*/", "", open(sys.argv[2]).read(), flags=re.S)
for n in sorted(set(re.findall(r"\b(dg[a-z0-9_]*)\s*\(", text))):
    f = getattr(lib, n)
    args = [0 if t in (ctypes.c_int, ctypes.c_uint, ctypes.c_longlong) else 0.0 if t is ctypes.c_double else None
            for t in f.argtypes]
    f(*args)
print("survived")
"""


def test_every_entry_point_survives_null_and_zero_arguments(tmp_path):
    """Every function of include/dg_b200.h called with NULL pointers and zero
    sizes (a null context, no mesh, no buffers) returns an error code (or, for
    the destroy calls and pointer getters, nothing) instead of dereferencing
    them; run in a child process so that a fault would fail this test."""
    import subprocess
    import sys
    script = tmp_path / "nulls.py"
    script.write_text(NULL_CHILD)
    r = subprocess.run([sys.executable, str(script), os.path.join(ROOT, "dg-mpi_b200"),
                        os.path.join(ROOT, "include", "dg_b200.h")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().endswith("survived")
