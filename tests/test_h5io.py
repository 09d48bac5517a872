"""Mesh and solution files in the reference's HDF5 schemas (host only).

The library's HDF5 subset reader is checked on the reference's own mesh files
(tests/golden/meshes, copied byte for byte, SHA-256 pinned) against an
independent test-side decoder and against the meshes' geometry; its writer's
files are decoded by the test-side decoder, which enforces the structure the
HDF5 library relies on; solution files written by ranks in either storage
layout (made by the test-side encoder) are read back in global element order;
corrupt files fail with an error, never a crash.
"""
import hashlib
import os

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401  (puts the package on sys.path)
import dg_b200
import h5_subset

MESHES = os.path.join(os.path.dirname(__file__), "golden", "meshes")
# nodes of each local face of a linear quadrilateral, x fastest
# (get_local_nodes_on_face_quadrilateral, src/numerics/basis/shape.cpp:125-152)
QUAD_FACE_NODES = [(0, 1), (1, 3), (3, 2), (2, 0)]


def test_mesh_fixtures_are_the_pinned_copies(golden):
    for name, meta in golden["mesh_files"].items():
        with open(os.path.join(MESHES, name), "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == meta["sha256"], name


@pytest.mark.parametrize("name", ["quad_1x1.h5", "quad_2x2.h5", "mpi_test_mesh.h5"])
def test_reader_agrees_with_independent_decoder_on_reference_files(name):
    path = os.path.join(MESHES, name)
    m = dg_b200.read_mesh_h5(path)
    ref = h5_subset.read(path)["datasets"]
    assert m.dim == int(ref["Dimension"]) and m.qorder == int(ref["QOrder"])
    assert np.array_equal(m.node_coords, ref["NodeCoords"])
    assert np.array_equal(m.elem_to_node_ids, ref["Elem2Nodes"])
    ifd = ref["IFaceData"]
    assert m.interior_faces.shape == (int(ref["nIFace"]), 8)
    assert np.array_equal(m.interior_faces[:, [1, 2, 3, 5, 6, 7]], ifd)
    assert not m.interior_faces[:, [0, 4]].any()
    assert m.elem_to_node_ids.shape == (int(ref["nElem"]), int(ref["nNodePerElem"]))


@pytest.mark.parametrize("name", ["quad_1x1.h5", "quad_2x2.h5"])
def test_reference_quad_meshes_faces_match_geometrically(name):
    """Both sides of every interior face hold the same two nodes, up to a
    periodic shift by the domain's extent."""
    m = dg_b200.read_mesh_h5(os.path.join(MESHES, name))
    assert (m.dim, m.qorder, m.elem_to_node_ids.shape[1]) == (2, 1, 4)
    x = m.node_coords
    ext = x.max(0) - x.min(0)
    for row in m.interior_faces:
        pts = []
        for eid, lf in ((row[1], row[2]), (row[5], row[6])):
            nodes = m.elem_to_node_ids[eid][list(QUAD_FACE_NODES[lf])]
            pts.append(x[nodes])
        shift = pts[0].mean(0) - pts[1].mean(0)
        k = np.round(shift / ext)
        assert np.allclose(shift, k * ext) and np.count_nonzero(k) <= 1
        a = sorted(map(tuple, np.round(pts[0] - k * ext, 12)))
        b = sorted(map(tuple, np.round(pts[1], 12)))
        assert a == b


def test_reference_triangle_mesh_neighbours_share_a_face():
    m = dg_b200.read_mesh_h5(os.path.join(MESHES, "mpi_test_mesh.h5"))
    assert m.elem_to_node_ids.shape == (242, 3) and m.interior_faces.shape == (343, 8)
    for row in m.interior_faces:
        shared = set(m.elem_to_node_ids[row[1]]) & set(m.elem_to_node_ids[row[5]])
        assert len(shared) == 2
    counts = np.bincount(m.interior_faces[:, [1, 5]].ravel(), minlength=242)
    assert counts.max() <= 3


def test_hex_mesh_round_trip_and_schema(tmp_path):
    m = dg_b200.periodic_box((3, 4, 5), (0.5, -1.0, 0.0), (1.0, 2.0, 3.0), rotate_seed=11)
    path = str(tmp_path / "cube.h5")
    dg_b200.write_mesh_h5(path, m)
    r = dg_b200.read_mesh_h5(path)
    assert (r.dim, r.qorder) == (3, 1)
    for a, b in ((r.node_coords, m.node_coords), (r.elem_to_node_ids, m.elem_to_node_ids),
                 (r.interior_faces, m.interior_faces)):
        assert np.array_equal(a, b)
    d = h5_subset.read(path)["datasets"]
    assert {k: int(d[k]) for k in ("Dimension", "QOrder", "nElem", "nNode", "nIFace", "nNodePerElem",
                                   "nNodePerFace", "nBFaceGroup")} == \
        {"Dimension": 3, "QOrder": 1, "nElem": 60, "nNode": m.node_coords.shape[0], "nIFace": 180,
         "nNodePerElem": 8, "nNodePerFace": 4, "nBFaceGroup": 0}
    assert d["Elem2Nodes"].dtype == np.int64 and d["IFaceData"].dtype == np.int64
    assert np.array_equal(d["IFaceData"], m.iface_data())


def test_solution_round_trip_and_writer_schema(tmp_path):
    m = dg_b200.periodic_box((2, 3, 2), (0, 0, 0), (1, 1, 1))
    U = np.random.default_rng(3).standard_normal((m.nelem, 64, 5))
    path = str(tmp_path / "data.h5")
    dg_b200.write_solution_h5(path, m, 3, U, 0.75)
    V, t = dg_b200.read_solution_h5(path)
    assert np.array_equal(U, V) and t == 0.75
    f = h5_subset.read(path)
    root = f["attrs"][""]
    assert {k: (int(v) if k != "Solver Final Time" else float(v)) for k, v in root.items()} == {
        "Number of Ranks": 1, "Number of Dimensions": 3, "Number of Elements": 12,
        "Number of Nodes": m.node_coords.shape[0], "Number of Nodes Per Element": 8, "Number of Basis Functions": 64,
        "Number of State Variables": 5, "Solver Final Time": 0.75, "Stored Layout": 1}
    assert root["Stored Layout"].dtype == np.int32 and root["Number of Elements"].dtype == np.uint32
    ds = f["datasets"]
    assert ds["Solution Coefficients"].shape == (12 * 64 * 5,)
    assert np.array_equal(ds["Solution Coefficients"], U.ravel())
    assert list(ds["Solution Coefficients_dims"]) == [12, 64, 5]
    assert list(ds["Solution Coefficients_offsets"]) == [0]
    oa = f["attrs"]["Solution Coefficients_offsets"]
    assert (int(oa["nDims"]), int(oa["nRanks"]), int(oa["totalSize"])) == (3, 1, 12 * 64 * 5)
    assert np.array_equal(ds["Element Global Node IDs"], m.elem_to_node_ids.ravel())
    assert np.array_equal(ds["Node Coordinates"], m.node_coords.ravel())
    assert list(ds["Number of Elements per Partition"]) == [12]
    for name in ("Local to Global Node ID", "Local to Global Element IDs"):
        assert np.array_equal(ds[name], np.arange(ds[name].size))


def _ranked_solution_file(path, U, parts, row_major, time=1.5):
    """A solution file written by len(parts) ranks (parts: each rank's global
    element ids), in the given storage layout (HDF5Wrapper.h:775-880)."""
    ne, nb, ns = U.shape
    blocks, offs, dims, ids = [], [], [], []
    at = 0
    for g in parts:
        blk = U[g] if row_major else np.transpose(U[g], (2, 1, 0))
        blocks.append(np.ascontiguousarray(blk).ravel())
        offs.append(at)
        at += blocks[-1].size
        dims += [len(g), nb, ns]
        ids.append(np.asarray(g, np.uint32))
    nr = len(parts)
    ds = {"Solution Coefficients": np.concatenate(blocks),
          "Solution Coefficients_offsets": np.array(offs, np.uint64),
          "Solution Coefficients_dims": np.array(dims, np.uint64),
          "Local to Global Element IDs": np.concatenate(ids),
          "Local to Global Element IDs_offsets": np.cumsum([0] + [len(g) for g in parts[:-1]]).astype(np.uint64),
          "Local to Global Element IDs_dims": np.array([len(g) for g in parts], np.uint64),
          "Number of Elements per Partition": np.array([len(g) for g in parts], np.uint32)}
    attrs = {"": {"Number of Ranks": np.uint32(nr), "Number of Elements": np.uint32(ne),
                  "Number of Basis Functions": np.uint32(nb), "Number of State Variables": np.uint32(ns),
                  "Solver Final Time": np.float64(time), "Stored Layout": np.int32(1 if row_major else 0)}}
    for name, nd, total in (("Solution Coefficients", 3, at), ("Local to Global Element IDs", 1, ne)):
        attrs[name + "_offsets"] = {"nDims": np.uint64(nd), "nRanks": np.int32(nr), "totalSize": np.uint64(total)}
    h5_subset.write(path, ds, attrs)


@pytest.mark.parametrize("row_major", [True, False])
def test_solution_reader_orders_rank_blocks_in_either_layout(tmp_path, row_major):
    rng = np.random.default_rng(5)
    U = rng.standard_normal((10, 8, 5))
    perm = rng.permutation(10)
    parts = [list(perm[:4]), list(perm[4:])]
    path = str(tmp_path / "ranked.h5")
    _ranked_solution_file(path, U, parts, row_major)
    V, t = dg_b200.read_solution_h5(path)
    assert t == 1.5 and np.array_equal(U, V)


def test_solution_reader_rejects_incomplete_element_sets(tmp_path):
    U = np.zeros((6, 8, 5))
    path = str(tmp_path / "dup.h5")
    _ranked_solution_file(path, U, [[0, 1, 2], [2, 3, 4]], True)
    with pytest.raises(dg_b200.DGError, match="permutation"):
        dg_b200.read_solution_h5(path)


def test_independent_encoder_file_reads_in_library(tmp_path):
    """The test-side encoder's mesh file (a different B-tree fill) reads the same."""
    m = dg_b200.periodic_box((2, 2, 3), (0, 0, 0), (1, 1, 1), rotate_seed=2)
    path = str(tmp_path / "enc.h5")
    scal = lambda v: np.array(v, np.int64)
    h5_subset.write(path, {"Dimension": scal(3), "QOrder": scal(1), "nElem": scal(m.nelem),
                           "nNode": scal(m.node_coords.shape[0]), "nIFace": scal(m.interior_faces.shape[0]),
                           "nNodePerElem": scal(8), "nNodePerFace": scal(4), "NodeCoords": m.node_coords,
                           "Elem2Nodes": m.elem_to_node_ids.astype(np.int64),
                           "IFaceData": m.iface_data().astype(np.int64)})
    r = dg_b200.read_mesh_h5(path)
    assert np.array_equal(r.interior_faces, m.interior_faces) and np.array_equal(r.node_coords, m.node_coords)


def test_corrupt_files_fail_cleanly(tmp_path):
    good = os.path.join(MESHES, "quad_2x2.h5")
    data = open(good, "rb").read()
    bad = tmp_path / "bad.h5"
    rng = np.random.default_rng(9)
    for cut in sorted(set(rng.integers(0, len(data), 40).tolist()) | {0, 8, 95, 96, 500}):
        bad.write_bytes(data[:cut])
        with pytest.raises(dg_b200.DGError):
            dg_b200.read_mesh_h5(str(bad))
    outcomes = 0
    for _ in range(200):
        b = bytearray(data)
        for pos in rng.integers(0, len(b), 4):
            b[pos] = int(rng.integers(0, 256))
        bad.write_bytes(bytes(b))
        try:
            dg_b200.read_mesh_h5(str(bad))
        except dg_b200.DGError:
            outcomes += 1
    assert outcomes > 0
    bad.write_bytes(b"not an hdf5 file" * 10)
    with pytest.raises(dg_b200.DGError, match="not an HDF5 file"):
        dg_b200.read_mesh_h5(str(bad))
    with pytest.raises(dg_b200.DGError, match="cannot open"):
        dg_b200.read_mesh_h5(str(tmp_path / "missing.h5"))


def test_solution_sizes_must_match_the_stored_coefficients(tmp_path):
    """The sizes query of a solution file checks the element, basis and
    variable counts against the stored coefficients, so a caller never
    allocates from a corrupt count."""
    m = dg_b200.periodic_box((2, 2, 2))
    U = np.random.default_rng(0).standard_normal((8, 27, 5))
    good = tmp_path / "sol.h5"
    dg_b200.write_solution_h5(str(good), m, 2, U, 0.5)
    data = bytearray(good.read_bytes())
    import struct
    # the root attribute "Number of Elements" holds 8 as an 8-byte integer right after its name
    at = data.find(b"Number of Elements")
    assert at > 0
    pos = data.find(struct.pack("<q", 8), at)
    assert pos > 0
    data[pos:pos + 8] = struct.pack("<q", 486539272)
    bad = tmp_path / "bad.h5"
    bad.write_bytes(bytes(data))
    with pytest.raises(dg_b200.DGError, match="disagree with the stored coefficients"):
        dg_b200.read_solution_h5(str(bad))


def test_mesh_counts_must_match_the_stored_arrays(tmp_path):
    """The sizes query of a mesh file checks nNode, nElem and nIFace against
    the stored arrays before a caller allocates from them (a file written by
    the test-side encoder with every array intact and one count wrong)."""
    mesh = dg_b200.periodic_box((2, 2, 2))
    good = tmp_path / "mesh.h5"
    dg_b200.write_mesh_h5(str(good), mesh)
    ds = h5_subset.read(str(good))["datasets"]
    for key in ("nElem", "nNode", "nIFace"):
        bad_ds = dict(ds)
        bad_ds[key] = np.array(1 << 29, dtype=np.int64)
        bad = tmp_path / f"bad_{key}.h5"
        h5_subset.write(str(bad), bad_ds)
        with pytest.raises(dg_b200.DGError, match="disagree with the counts"):
            dg_b200.read_mesh_h5(str(bad))
    ok = tmp_path / "ok.h5"
    h5_subset.write(str(ok), ds)
    assert dg_b200.read_mesh_h5(str(ok)).elem_to_node_ids.shape == (8, 8)


def test_cyclic_group_btree_fails_cleanly(tmp_path):
    """A group B-tree node turned into an internal node whose child is itself
    (a cycle) is refused, not walked forever."""
    b = bytearray(open(os.path.join(MESHES, "quad_2x2.h5"), "rb").read())
    root = int.from_bytes(b[64:72], "little")
    stab = [m for t, m in h5_subset._messages(bytes(b), root) if t == 0x11][0]
    btree = int.from_bytes(stab[0:8], "little")
    assert b[btree:btree + 4] == b"TREE"
    b[btree + 5] = 1                                        # level 1: children are B-tree nodes
    b[btree + 32:btree + 40] = btree.to_bytes(8, "little")  # first child: the node itself
    bad = tmp_path / "cyclic.h5"
    bad.write_bytes(bytes(b))
    with pytest.raises(dg_b200.DGError, match="B-tree"):
        dg_b200.read_mesh_h5(str(bad))


def test_two_dimensional_mesh_is_refused_by_the_context_boundary():
    m = dg_b200.read_mesh_h5(os.path.join(MESHES, "quad_2x2.h5"))
    with pytest.raises(ValueError, match="3D meshes"):
        dg_b200.write_mesh_h5("/dev/null", m)
