"""Python binding of libdg_b200.so (the C ABI declared in include/dg_b200.h).

The library is the product: CUDA kernels for sm_100a behind a C ABI plus the
C++ host side (mesh, tables, initial conditions).  This module only marshals
numpy arrays through ctypes; it computes nothing itself and has no fallback:
if the shared library is missing or no GPU is present, the calls fail loudly.

Names follow the reference's vocabulary (IhmeGroup/DG-MPI): a *case* is one
mesh + order + physics setup, ``Uc`` is the solution-coefficient array
[ne][nb][5] (src/solver/base.h), ``res`` the residual of
Solver<3>::get_residual, ``interior_faces`` the [nface][8] connectivity of
src/mesh/mesh.h:280-284.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libdg_b200.so")

DG_OK = 0
DG_ERR_TIMEOUT = 4
ERROR_NAMES = {1: "DG_ERR_ARG", 2: "DG_ERR_CUDA", 3: "DG_ERR_NONPHYSICAL", 4: "DG_ERR_TIMEOUT",
               5: "DG_ERR_UNSUPPORTED", 6: "DG_ERR_NOMEM"}

FLUX = {"LaxFriedrichs": 0, "HLLC": 1}
PRECISION = {"fp64": 0, "mixed_fp32": 1}
# [InitialCondition] name -> DG_IC_* (include/dg_b200.h)
IC = {"Uniform": 0, "IsentropicVortex": 1, "Sphere": 2, "IsentropicVortexXY": 3, "TaylorGreen": 4}
# the 2D path's families: the reference's 2D vortex (data rho, u, v, p, strength),
# the x-y vortex at (x, y, 0), a uniform state of four conserved values
IC2D = {"Uniform": 0, "IsentropicVortex": 5, "IsentropicVortexXY": 3}


class DGError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


class _MeshDesc(ctypes.Structure):
    _fields_ = [("nnode", ctypes.c_int), ("node_coords", ctypes.POINTER(ctypes.c_double)),
                ("nelem", ctypes.c_int), ("elem_to_node_ids", ctypes.POINTER(ctypes.c_uint)),
                ("nface", ctypes.c_int), ("interior_faces", ctypes.POINTER(ctypes.c_uint)),
                ("rank", ctypes.c_int)]


class _CaseDesc(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int), ("flux", ctypes.c_int), ("gamma", ctypes.c_double),
                ("gas_constant", ctypes.c_double), ("precision", ctypes.c_int), ("device", ctypes.c_int)]


class _PartDesc(ctypes.Structure):
    _fields_ = [("nowned", ctypes.c_int), ("ninterior", ctypes.c_int), ("ghost_rank", ctypes.POINTER(ctypes.c_int)),
                ("ghost_elem", ctypes.POINTER(ctypes.c_int))]


# RK4 buffers (DG_BUF_*): the state, and the two stage buffers; stage s reads STAGE_INPUT[s]
BUF_U0, BUF_STAGE_A, BUF_STAGE_B = 0, 1, 2
STAGE_INPUT = {1: BUF_U0, 2: BUF_STAGE_A, 3: BUF_STAGE_B, 4: BUF_STAGE_A}

_lib = None


def library(path: str | None = None) -> ctypes.CDLL:
    """Load libdg_b200.so once (raises OSError if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    lib = ctypes.CDLL(path or LIB_PATH)
    dp = ctypes.POINTER(ctypes.c_double)
    up = ctypes.POINTER(ctypes.c_uint)
    ip = ctypes.POINTER(ctypes.c_int)
    vp = ctypes.c_void_p
    sig = {
        "dg_create": (ctypes.c_int, [ctypes.POINTER(_CaseDesc), ctypes.POINTER(_MeshDesc), ctypes.POINTER(vp)]),
        "dg_destroy": (None, [vp]),
        "dg_last_error": (ctypes.c_char_p, [vp]),
        "dg_num_basis": (ctypes.c_int, [vp]),
        "dg_num_elements": (ctypes.c_int, [vp]),
        "dg_set_state": (ctypes.c_int, [vp, dp]),
        "dg_get_state": (ctypes.c_int, [vp, dp]),
        "dg_residual": (ctypes.c_int, [vp, dp]),
        "dg_mass_inverse_residual": (ctypes.c_int, [vp, ctypes.c_double, dp]),
        "dg_rk4_steps": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "dg_rk4_steps_timed": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, dp]),
        "dg_fe_steps": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "dg_project_ic": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, dp]),
        "dg_l2_error": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, dp]),
        "dg_kinetic_energy": (ctypes.c_int, [vp, dp]),
        "dg_kinetic_energy_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, vp, vp, vp, vp]),
        "dg_total_volume": (ctypes.c_int, [vp, dp]),
        "dg_status": (ctypes.c_int, [vp, up]),
        "dg_sync": (ctypes.c_int, [vp]),
        "dg_probe_bounded_wait": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong, ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_longlong)]),
        "dg_device_state": (vp, [vp]),
        "dg_mesh_periodic_box": (ctypes.c_int, [ip, dp, dp, ctypes.c_uint, ip, dp, ip, up, ip, up]),
        "dg_cfl_time_step": (ctypes.c_int, [vp, dp, ctypes.c_double, dp]),
        "dg_gauss_legendre": (ctypes.c_int, [ctypes.c_int, dp, dp]),
        "dg_face_orientation_order": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ip]),
        "dg_basis_tables": (ctypes.c_int, [ctypes.c_int, dp, dp, dp]),
        "dg_num_stage_variants": (ctypes.c_int, [ctypes.c_int]),
        "dg_stage_variant_info": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ip, ip, ip, ip]),
        "dg_stage_variant_flags": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ip]),
        "dg_set_stage_variant": (ctypes.c_int, [vp, ctypes.c_int]),
        "dg_set_stage_chunks": (ctypes.c_int, [vp, ctypes.c_int]),
        "dg_get_stage_chunks": (ctypes.c_int, [vp]),
        "dg_get_stage_variant": (ctypes.c_int, [vp]),
        "dg_tune_stage": (ctypes.c_int, [vp, ctypes.c_int, ip, dp]),
        "dg_create_partitioned": (ctypes.c_int, [ctypes.POINTER(_CaseDesc), ctypes.POINTER(_MeshDesc),
                                                 ctypes.POINTER(_PartDesc), ctypes.POINTER(vp)]),
        "dg_partition_periodic_box": (ctypes.c_int, [ip, dp, dp, ctypes.c_uint, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                     ip, dp, ip, up, ip, up, ip, ip, ip, ip, ip]),
        "dg_halo_plan": (ctypes.c_int, [ctypes.POINTER(_MeshDesc), ctypes.POINTER(_PartDesc), ip, ip, ip, ip, ip,
                                        ip, ip, ip, ip]),
        "dg_halo_num_peers": (ctypes.c_int, [vp]),
        "dg_halo_peer": (ctypes.c_int, [vp, ctypes.c_int, ip, ip, ip]),
        "dg_halo_slice_doubles": (ctypes.c_int, [vp]),
        "dg_halo_pack": (ctypes.c_int, [vp, ctypes.c_int, vp, vp]),
        "dg_halo_unpack": (ctypes.c_int, [vp, ctypes.c_int, vp, vp]),
        "dg_rk4_stage": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
        "dg_stream": (vp, [vp]),
        "dg_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_CaseDesc), ctypes.POINTER(_MeshDesc),
                                           ctypes.POINTER(vp)]),
        "dg_batch_destroy": (None, [vp]),
        "dg_batch_last_error": (ctypes.c_char_p, [vp]),
        "dg_batch_num_groups": (ctypes.c_int, [vp]),
        "dg_batch_group_info": (ctypes.c_int, [vp, ctypes.c_int, ip, ip, ip, ip]),
        "dg_batch_case_info": (ctypes.c_int, [vp, ctypes.c_int, ip, ip, ip, dp]),
        "dg_batch_set_state": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "dg_batch_get_state": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "dg_batch_project_ic": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, dp]),
        "dg_batch_cfl_time_step": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_double, dp]),
        "dg_batch_set_time_step": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double]),
        "dg_batch_rk4_steps": (ctypes.c_int, [vp, ctypes.c_int]),
        "dg_batch_rk4_steps_timed": (ctypes.c_int, [vp, ctypes.c_int, dp]),
        "dg_batch_tune": (ctypes.c_int, [vp, ctypes.c_int]),
        "dg_batch_set_launch_mode": (ctypes.c_int, [vp, ctypes.c_int]),
        "dg_batch_get_launch_mode": (ctypes.c_int, [vp]),
        "dg_batch_l2_error": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, dp]),
        "dg_batch_status": (ctypes.c_int, [vp, up]),
        "dg_mesh_read_h5": (ctypes.c_int, [ctypes.c_char_p, ip, ip, ip, ip, dp, ip, up, ip, up]),
        "dg_mesh_write_h5": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_MeshDesc)]),
        "dg_solution_write_h5": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_MeshDesc), ctypes.c_int, dp,
                                                ctypes.c_double]),
        "dg_solution_read_h5": (ctypes.c_int, [ctypes.c_char_p, ip, ip, ip, dp, dp]),
        "dg2d_create": (ctypes.c_int, [ctypes.POINTER(_CaseDesc), ctypes.POINTER(_MeshDesc), ctypes.POINTER(vp)]),
        "dg2d_destroy": (None, [vp]),
        "dg2d_last_error": (ctypes.c_char_p, [vp]),
        "dg2d_num_basis": (ctypes.c_int, [vp]),
        "dg2d_set_state": (ctypes.c_int, [vp, dp]),
        "dg2d_get_state": (ctypes.c_int, [vp, dp]),
        "dg2d_residual": (ctypes.c_int, [vp, dp]),
        "dg2d_rk4_steps": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "dg2d_rk4_steps_timed": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int, dp]),
        "dg2d_fe_steps": (ctypes.c_int, [vp, ctypes.c_double, ctypes.c_int]),
        "dg2d_project_ic": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, dp]),
        "dg2d_l2_error": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double, dp]),
        "dg2d_status": (ctypes.c_int, [vp, up]),
        "dg_mesh2d_periodic_box": (ctypes.c_int, [ip, dp, dp, ctypes.c_uint, ip, dp, ip, up, ip, up]),
        "dg2d_solution_write_h5": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_MeshDesc), ctypes.c_int, dp,
                                                  ctypes.c_double]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _uptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint))


@dataclass
class Mesh:
    """Hex mesh in the reference's in-memory form (src/mesh/mesh.h).  A mesh
    read from a file may have another dimension or element type (dim, the
    file's QOrder); contexts take dim 3, qorder 1, 8-node hexahedra."""
    node_coords: np.ndarray      # [nnode][dim] float64
    elem_to_node_ids: np.ndarray  # [nelem][nodes per element] uint32
    interior_faces: np.ndarray    # [nface][8] uint32
    dim: int = 3
    qorder: int = 1

    @property
    def nelem(self) -> int:
        return int(self.elem_to_node_ids.shape[0])

    def iface_data(self) -> np.ndarray:
        """The [nface][6] IFaceData of the mesh file (mesh/mesh.cpp:144-160)."""
        f = self.interior_faces
        return np.ascontiguousarray(f[:, [1, 2, 3, 5, 6, 7]].astype(np.int32))


def periodic_box(n, x0=(0.0, 0.0, 0.0), length=(1.0, 1.0, 1.0), rotate_seed: int = 0) -> Mesh:
    """Uniform periodic hex box from the library's host-side generator."""
    lib = library()
    n_arr = (ctypes.c_int * 3)(*[int(v) for v in n])
    x_arr = (ctypes.c_double * 3)(*[float(v) for v in x0])
    l_arr = (ctypes.c_double * 3)(*[float(v) for v in length])
    nn, ne, nf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = lib.dg_mesh_periodic_box(n_arr, x_arr, l_arr, ctypes.c_uint(rotate_seed), ctypes.byref(nn), None,
                                  ctypes.byref(ne), None, ctypes.byref(nf), None)
    if rc:
        raise DGError(rc, "dg_mesh_periodic_box: bad box")
    coords = np.zeros((nn.value, 3), np.float64)
    e2n = np.zeros((ne.value, 8), np.uint32)
    faces = np.zeros((nf.value, 8), np.uint32)
    rc = lib.dg_mesh_periodic_box(n_arr, x_arr, l_arr, ctypes.c_uint(rotate_seed), ctypes.byref(nn), _dptr(coords),
                                  ctypes.byref(ne), _uptr(e2n), ctypes.byref(nf), _uptr(faces))
    if rc:
        raise DGError(rc, "dg_mesh_periodic_box failed")
    return Mesh(coords, e2n, faces)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


@dataclass
class Partition:
    """One rank's share of a partitioned mesh: owned elements [0, nowned) (the
    first ninterior without ghost neighbours), then ghosts, each with its
    owner rank and its local id there (dg_part_desc)."""
    rank: int
    nowned: int
    ninterior: int
    ghost_rank: np.ndarray   # int32 [nghost]
    ghost_elem: np.ndarray   # int32 [nghost]
    global_elem: np.ndarray  # int32 [nowned + nghost], ids in the unpartitioned mesh

    def desc(self) -> _PartDesc:
        self.ghost_rank = np.ascontiguousarray(self.ghost_rank, np.int32)
        self.ghost_elem = np.ascontiguousarray(self.ghost_elem, np.int32)
        return _PartDesc(self.nowned, self.ninterior, _iptr(self.ghost_rank), _iptr(self.ghost_elem))


def partition_periodic_box(n, x0, length, nparts: int, part: int, axis: int = 2, rotate_seed: int = 0):
    """Slab `part` of `nparts` along `axis` of periodic_box(n, x0, length): (Mesh, Partition)."""
    lib = library()
    n_arr = (ctypes.c_int * 3)(*[int(v) for v in n])
    x_arr = (ctypes.c_double * 3)(*[float(v) for v in x0])
    l_arr = (ctypes.c_double * 3)(*[float(v) for v in length])
    nn, ne, nf, no, ni = (ctypes.c_int() for _ in range(5))
    args = (n_arr, x_arr, l_arr, ctypes.c_uint(rotate_seed), nparts, part, axis)
    rc = lib.dg_partition_periodic_box(*args, ctypes.byref(nn), None, ctypes.byref(ne), None, ctypes.byref(nf), None,
                                       ctypes.byref(no), ctypes.byref(ni), None, None, None)
    if rc:
        raise DGError(rc, "dg_partition_periodic_box: bad arguments")
    coords = np.zeros((nn.value, 3), np.float64)
    e2n = np.zeros((ne.value, 8), np.uint32)
    faces = np.zeros((nf.value, 8), np.uint32)
    ng = ne.value - no.value
    gr, ge, gl = np.zeros(ng, np.int32), np.zeros(ng, np.int32), np.zeros(ne.value, np.int32)
    rc = lib.dg_partition_periodic_box(*args, ctypes.byref(nn), _dptr(coords), ctypes.byref(ne), _uptr(e2n),
                                       ctypes.byref(nf), _uptr(faces), ctypes.byref(no), ctypes.byref(ni), _iptr(gr),
                                       _iptr(ge), _iptr(gl))
    if rc:
        raise DGError(rc, "dg_partition_periodic_box failed")
    return Mesh(coords, e2n, faces), Partition(part, no.value, ni.value, gr, ge, gl)


def _path(path) -> bytes:
    return os.fsencode(os.fspath(path))


def read_mesh_h5(path) -> Mesh:
    """A mesh file of the reference's format (Mesh::read_mesh,
    src/mesh/mesh.cpp:79-204) through dg_mesh_read_h5."""
    lib = library()
    d, q, npe, nn, ne, nf = (ctypes.c_int() for _ in range(6))
    args = [ctypes.byref(v) for v in (d, q, npe, nn)]
    rc = lib.dg_mesh_read_h5(_path(path), *args, None, ctypes.byref(ne), None, ctypes.byref(nf), None)
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())
    coords = np.zeros((nn.value, d.value), np.float64)
    e2n = np.zeros((ne.value, npe.value), np.uint32)
    faces = np.zeros((nf.value, 8), np.uint32)
    rc = lib.dg_mesh_read_h5(_path(path), *args, _dptr(coords), ctypes.byref(ne), _uptr(e2n), ctypes.byref(nf),
                             _uptr(faces))
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())
    return Mesh(coords, e2n, faces, d.value, q.value)


def write_mesh_h5(path, mesh: Mesh):
    """Writes a hexahedral mesh in the reference's mesh-file format (dg_mesh_write_h5)."""
    lib = library()
    keep = []
    md = _mesh_desc(mesh, 0, keep)
    rc = lib.dg_mesh_write_h5(_path(path), ctypes.byref(md))
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())


def write_solution_h5(path, mesh: Mesh, order: int, Uc: np.ndarray, time: float = 0.0):
    """Writes Uc[ne][nb][5] in the reference writer's data.h5 schema
    (Writer::write, src/io/writer.cpp:10-64) through dg_solution_write_h5."""
    lib = library()
    keep = []
    md = _mesh_desc(mesh, 0, keep)
    U = np.ascontiguousarray(Uc, np.float64)
    if U.size != mesh.nelem * (order + 1) ** 3 * 5:
        raise ValueError("Uc does not hold a state of this mesh and order")
    rc = lib.dg_solution_write_h5(_path(path), ctypes.byref(md), int(order), _dptr(U), float(time))
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())


def read_solution_h5(path):
    """(Uc [ne][nb][ns], time) from a data.h5 of the reference writer's schema
    (Solver::read_in_coefficients, src/solver/base.cpp:234-279)."""
    lib = library()
    ne, nb, ns, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    rc = lib.dg_solution_read_h5(_path(path), ctypes.byref(ne), ctypes.byref(nb), ctypes.byref(ns), ctypes.byref(t),
                                 None)
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())
    U = np.zeros((ne.value, nb.value, ns.value), np.float64)
    rc = lib.dg_solution_read_h5(_path(path), ctypes.byref(ne), ctypes.byref(nb), ctypes.byref(ns), ctypes.byref(t),
                                 _dptr(U))
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())
    return U, t.value


def _mesh_desc(mesh: Mesh, rank: int, keep: list) -> _MeshDesc:
    c = np.ascontiguousarray(mesh.node_coords, np.float64)
    e = np.ascontiguousarray(mesh.elem_to_node_ids, np.uint32)
    f = np.ascontiguousarray(mesh.interior_faces, np.uint32)
    if c.ndim != 2 or c.shape[1] != 3 or e.ndim != 2 or e.shape[1] != 8 or f.ndim != 2 or f.shape[1] != 8:
        raise ValueError("the C ABI takes 3D meshes of 8-node hexahedra (node_coords [n][3], "
                         "elem_to_node_ids [ne][8], interior_faces [nf][8])")
    keep += [c, e, f]
    return _MeshDesc(c.shape[0], _dptr(c), e.shape[0], _uptr(e), f.shape[0], _uptr(f), rank)


def halo_plan(mesh: Mesh, part: Partition):
    """Host-side halo plan (dg_halo_plan): ([(peer rank, offset, count)], send (elem, face) [nslices][2],
    recv (ghost elem, face) [nslices][2])."""
    lib = library()
    keep = []
    md = _mesh_desc(mesh, part.rank, keep)
    pd = part.desc()
    npeer, nsl = ctypes.c_int(), ctypes.c_int()
    rc = lib.dg_halo_plan(ctypes.byref(md), ctypes.byref(pd), ctypes.byref(npeer), None, None, None, ctypes.byref(nsl),
                          None, None, None, None)
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())
    pr, po, pc = (np.zeros(npeer.value, np.int32) for _ in range(3))
    se, sf, re_, rf = (np.zeros(nsl.value, np.int32) for _ in range(4))
    rc = lib.dg_halo_plan(ctypes.byref(md), ctypes.byref(pd), ctypes.byref(npeer), _iptr(pr), _iptr(po), _iptr(pc),
                          ctypes.byref(nsl), _iptr(se), _iptr(sf), _iptr(re_), _iptr(rf))
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())
    peers = [(int(a), int(b), int(c)) for a, b, c in zip(pr, po, pc)]
    return peers, np.stack([se, sf], 1), np.stack([re_, rf], 1)


class Case:
    """One DG case on one GPU (a dg_ctx); with `part`, one rank's share of a
    partitioned mesh (dg_create_partitioned), whose ghost slices the caller
    exchanges through halo_pack / halo_unpack between rk4_stage calls."""

    def __init__(self, mesh: Mesh, order: int, flux: str = "LaxFriedrichs", gamma: float = 1.4,
                 gas_constant: float = 287.05, precision: str = "fp64", device: int = 0,
                 part: Partition | None = None):
        self._lib = library()
        self.mesh = mesh
        self.order = order
        self.nb = (order + 1) ** 3
        self.ne = mesh.nelem if part is None else part.nowned
        self.gamma = gamma
        self.part = part
        keep = []
        md = _mesh_desc(mesh, 0 if part is None else part.rank, keep)
        cd = _CaseDesc(order, FLUX[flux], gamma, gas_constant, PRECISION[precision], device)
        ctx = ctypes.c_void_p()
        if part is None:
            rc = self._lib.dg_create(ctypes.byref(cd), ctypes.byref(md), ctypes.byref(ctx))
        else:
            pd = part.desc()
            rc = self._lib.dg_create_partitioned(ctypes.byref(cd), ctypes.byref(md), ctypes.byref(pd), ctypes.byref(ctx))
        if rc:
            raise DGError(rc, self._lib.dg_last_error(None).decode())
        self._ctx = ctx

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int):
        if rc:
            raise DGError(rc, self._lib.dg_last_error(self._ctx).decode())

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.dg_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _state_array(self) -> np.ndarray:
        return np.empty((self.ne, self.nb, 5), np.float64)

    # -- the path ------------------------------------------------------------
    def set_state(self, Uc: np.ndarray):
        Uc = np.ascontiguousarray(Uc, np.float64)
        assert Uc.shape == (self.ne, self.nb, 5)
        self._check(self._lib.dg_set_state(self._ctx, _dptr(Uc)))

    def set_state_ptr(self, host_ptr: int):
        """Upload from a host buffer given by address (e.g. a pinned tensor)."""
        self._check(self._lib.dg_set_state(self._ctx, ctypes.cast(host_ptr, ctypes.POINTER(ctypes.c_double))))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        out = self._state_array() if out is None else out
        self._check(self._lib.dg_get_state(self._ctx, _dptr(out)))
        return out

    def get_state_ptr(self, host_ptr: int):
        self._check(self._lib.dg_get_state(self._ctx, ctypes.cast(host_ptr, ctypes.POINTER(ctypes.c_double))))

    def residual(self) -> np.ndarray:
        out = self._state_array()
        self._check(self._lib.dg_residual(self._ctx, _dptr(out)))
        return out

    def mass_inverse_residual(self, dt: float) -> np.ndarray:
        out = self._state_array()
        self._check(self._lib.dg_mass_inverse_residual(self._ctx, dt, _dptr(out)))
        return out

    def rk4(self, dt: float, nsteps: int):
        self._check(self._lib.dg_rk4_steps(self._ctx, dt, int(nsteps)))

    def rk4_timed(self, dt: float, nsteps: int) -> float:
        """RK4 steps; returns their device time in ms (CUDA events on the kernels' stream)."""
        ms = ctypes.c_double()
        self._check(self._lib.dg_rk4_steps_timed(self._ctx, dt, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def fe(self, dt: float, nsteps: int):
        self._check(self._lib.dg_fe_steps(self._ctx, dt, int(nsteps)))

    def project_ic(self, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        out = self._state_array()
        self._check(self._lib.dg_project_ic(self._ctx, IC[name], _dptr(d) if d.size else None, d.size, t, _dptr(out)))
        return out

    def l2_error(self, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        out = np.zeros(5, np.float64)
        self._check(self._lib.dg_l2_error(self._ctx, IC[name], _dptr(d) if d.size else None, d.size, t, _dptr(out)))
        return out

    def kinetic_energy(self) -> float:
        v = ctypes.c_double()
        self._check(self._lib.dg_kinetic_energy(self._ctx, ctypes.byref(v)))
        return v.value

    def total_volume(self) -> float:
        v = ctypes.c_double()
        self._check(self._lib.dg_total_volume(self._ctx, ctypes.byref(v)))
        return v.value

    def status(self) -> int:
        v = ctypes.c_uint()
        self._check(self._lib.dg_status(self._ctx, ctypes.byref(v)))
        return v.value

    def sync(self):
        self._check(self._lib.dg_sync(self._ctx))

    def cfl_time_step(self, Uc: np.ndarray, cfl: float) -> float:
        Uc = np.ascontiguousarray(Uc, np.float64)
        v = ctypes.c_double()
        self._check(self._lib.dg_cfl_time_step(self._ctx, _dptr(Uc), cfl, ctypes.byref(v)))
        return v.value

    def device_state_ptr(self) -> int:
        return int(self._lib.dg_device_state(self._ctx) or 0)

    # -- partitioned cases ---------------------------------------------------
    def halo_peers(self):
        """[(peer rank, slice offset, slice count)] of this rank's halo."""
        out = []
        for i in range(self._lib.dg_halo_num_peers(self._ctx)):
            r, o, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            self._check(self._lib.dg_halo_peer(self._ctx, i, ctypes.byref(r), ctypes.byref(o), ctypes.byref(c)))
            out.append((r.value, o.value, c.value))
        return out

    def halo_slice_doubles(self) -> int:
        return self._lib.dg_halo_slice_doubles(self._ctx)

    def halo_pack(self, buf: int, d_send: int, stream: int = 0):
        self._check(self._lib.dg_halo_pack(self._ctx, buf, ctypes.c_void_p(d_send), ctypes.c_void_p(stream or None)))

    def halo_unpack(self, buf: int, d_recv: int, stream: int = 0):
        self._check(self._lib.dg_halo_unpack(self._ctx, buf, ctypes.c_void_p(d_recv), ctypes.c_void_p(stream or None)))

    def rk4_stage(self, stage: int, dt: float, rng: int = 0):
        """Queue RK4 stage 1..4 on the context's stream over all owned (0), interior (1) or boundary (2) elements."""
        self._check(self._lib.dg_rk4_stage(self._ctx, int(stage), float(dt), int(rng)))

    def stream_ptr(self) -> int:
        return int(self._lib.dg_stream(self._ctx) or 0)

    # -- launch variants ---------------------------------------------------
    def stage_variants(self):
        """[(elements per CTA, threads per CTA, variable groups, precision, options)] compiled for this
        order; options is "" or a "+"-joined subset of "pz" (groups' pencils in one phase), "sb"
        (single coefficient buffer), "uf" (unfused volume), "rs" (row-split traces and lifts),
        "k1" (one face-flux point per thread), "ge" (general trilinear geometry: the variants that
        non-affine meshes run), "fx" (each face's flux once, from a face kernel launched before the
        stage kernel), "tc" (the tensor-core kernel: split products on tcgen05 for the volume
        integral), "mg" (the face lifts added inside the inverse mass's first pass), and "mb<n>"
        when the variant asks the compiler for n resident CTAs per SM."""
        out = []
        for v in range(self._lib.dg_num_stage_variants(self.order)):
            E, NT, G, pr, fl = (ctypes.c_int() for _ in range(5))
            self._lib.dg_stage_variant_info(self.order, v, ctypes.byref(E), ctypes.byref(NT), ctypes.byref(G),
                                            ctypes.byref(pr))
            self._lib.dg_stage_variant_flags(self.order, v, ctypes.byref(fl))
            opts = "+".join(n for b, n in ((1, "pz"), (2, "sb"), (4, "uf"), (8, "rs"), (16, "k1"), (32, "ge"), (64, "fx"),
                                           (128, "tc"), (4096, "mg")) if fl.value & b)
            if (fl.value >> 8) & 15:
                opts += ("+" if opts else "") + "mb%d" % ((fl.value >> 8) & 15)
            out.append((E.value, NT.value, G.value, "mixed_fp32" if pr.value == 1 else "fp64", opts))
        return out

    @property
    def stage_variant(self) -> int:
        return self._lib.dg_get_stage_variant(self._ctx)

    @stage_variant.setter
    def stage_variant(self, v: int):
        self._check(self._lib.dg_set_stage_variant(self._ctx, int(v)))

    @property
    def stage_chunks(self) -> int:
        """Element chunks per RK stage of the RK4 graph (dg_set_stage_chunks)."""
        return self._lib.dg_get_stage_chunks(self._ctx)

    @stage_chunks.setter
    def stage_chunks(self, n: int):
        self._check(self._lib.dg_set_stage_chunks(self._ctx, int(n)))

    def tune_stage(self, reps: int = 3):
        """Times every variant on this case (state unchanged), selects the fastest.
        Returns (best index, [ms per stage launch for each variant])."""
        n = self._lib.dg_num_stage_variants(self.order)
        ms = np.zeros(n, np.float64)
        best = ctypes.c_int()
        self._check(self._lib.dg_tune_stage(self._ctx, int(reps), ctypes.byref(best), _dptr(ms)))
        return best.value, ms.tolist()


class Batch:
    """An ensemble of independent cases advanced together (a dg_batch).

    ``cases`` is a sequence of (mesh, order) pairs; flux, gamma, gas constant,
    precision and device apply to all of them.  Cases of the same order share
    one stage launch per RK stage; every case has its own time step."""

    def __init__(self, cases, flux: str = "LaxFriedrichs", gamma: float = 1.4, gas_constant: float = 287.05,
                 precision: str = "fp64", device: int = 0):
        self._lib = library()
        self.orders = [int(o) for _, o in cases]
        self.nelem = [m.nelem for m, _ in cases]
        self._keep = []
        mds = (_MeshDesc * len(cases))()
        cds = (_CaseDesc * len(cases))()
        for i, (mesh, order) in enumerate(cases):
            c = np.ascontiguousarray(mesh.node_coords, np.float64)
            e = np.ascontiguousarray(mesh.elem_to_node_ids, np.uint32)
            f = np.ascontiguousarray(mesh.interior_faces, np.uint32)
            self._keep += [c, e, f]
            mds[i] = _MeshDesc(c.shape[0], _dptr(c), e.shape[0], _uptr(e), f.shape[0], _uptr(f), 0)
            cds[i] = _CaseDesc(int(order), FLUX[flux], gamma, gas_constant, PRECISION[precision], device)
        h = ctypes.c_void_p()
        rc = self._lib.dg_batch_create(len(cases), cds, mds, ctypes.byref(h))
        self._keep = None  # the library copied what it needs
        if rc:
            raise DGError(rc, self._lib.dg_batch_last_error(None).decode())
        self._b = h

    def _check(self, rc: int):
        if rc:
            raise DGError(rc, self._lib.dg_batch_last_error(self._b).decode())

    def close(self):
        if getattr(self, "_b", None):
            self._lib.dg_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.orders)

    def _state_array(self, c: int) -> np.ndarray:
        return np.empty((self.nelem[c], (self.orders[c] + 1) ** 3, 5), np.float64)

    def groups(self):
        """[(order, cases, elements, stage variant)] per group."""
        out = []
        for g in range(self._lib.dg_batch_num_groups(self._b)):
            o, n, e, v = (ctypes.c_int() for _ in range(4))
            self._check(self._lib.dg_batch_group_info(self._b, g, ctypes.byref(o), ctypes.byref(n), ctypes.byref(e),
                                                      ctypes.byref(v)))
            out.append((o.value, n.value, e.value, v.value))
        return out

    def set_state(self, c: int, Uc: np.ndarray):
        Uc = np.ascontiguousarray(Uc, np.float64)
        assert Uc.shape == self._state_array(c).shape
        self._check(self._lib.dg_batch_set_state(self._b, c, _dptr(Uc)))

    def get_state(self, c: int) -> np.ndarray:
        out = self._state_array(c)
        self._check(self._lib.dg_batch_get_state(self._b, c, _dptr(out)))
        return out

    def project_ic(self, c: int, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        out = self._state_array(c)
        self._check(self._lib.dg_batch_project_ic(self._b, c, IC[name], _dptr(d) if d.size else None, d.size, t,
                                                  _dptr(out)))
        return out

    def cfl_time_step(self, c: int, Uc: np.ndarray, cfl: float) -> float:
        Uc = np.ascontiguousarray(Uc, np.float64)
        v = ctypes.c_double()
        self._check(self._lib.dg_batch_cfl_time_step(self._b, c, _dptr(Uc), cfl, ctypes.byref(v)))
        return v.value

    def set_time_step(self, c: int, dt: float):
        self._check(self._lib.dg_batch_set_time_step(self._b, c, float(dt)))

    def rk4(self, nsteps: int):
        self._check(self._lib.dg_batch_rk4_steps(self._b, int(nsteps)))

    def rk4_timed(self, nsteps: int) -> float:
        ms = ctypes.c_double()
        self._check(self._lib.dg_batch_rk4_steps_timed(self._b, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def tune(self, reps: int = 2):
        self._check(self._lib.dg_batch_tune(self._b, int(reps)))

    @property
    def single_launch(self) -> bool:
        """True when each RK stage is one launch over all groups (possible when every
        group has order 1..5 on affine elements), False for one launch per group (the
        default; tune() keeps the faster of the two)."""
        return self._lib.dg_batch_get_launch_mode(self._b) == 1

    @single_launch.setter
    def single_launch(self, on: bool):
        self._check(self._lib.dg_batch_set_launch_mode(self._b, 1 if on else 0))

    def l2_error(self, c: int, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        out = np.zeros(5, np.float64)
        self._check(self._lib.dg_batch_l2_error(self._b, c, IC[name], _dptr(d) if d.size else None, d.size, t,
                                                _dptr(out)))
        return out

    def status(self) -> int:
        v = ctypes.c_uint()
        self._check(self._lib.dg_batch_status(self._b, ctypes.byref(v)))
        return v.value


def gauss_legendre(n: int):
    """n-point Gauss-Legendre rule of the host side."""
    x, w = np.zeros(n), np.zeros(n)
    rc = library().dg_gauss_legendre(n, _dptr(x), _dptr(w))
    if rc:
        raise DGError(rc, "dg_gauss_legendre")
    return x, w


def face_orientation_order(orient: int, npts: int) -> np.ndarray:
    out = np.zeros(npts, np.int32)
    rc = library().dg_face_orientation_order(orient, npts, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc:
        raise DGError(rc, "dg_face_orientation_order")
    return out


def basis_tables(p: int):
    """(B[m][n], D[m][n], Minv[n][n]) 1D tables of order p."""
    n, m = p + 1, p + 2
    B, D, Mi = np.zeros((m, n)), np.zeros((m, n)), np.zeros((n, n))
    rc = library().dg_basis_tables(p, _dptr(B), _dptr(D), _dptr(Mi))
    if rc:
        raise DGError(rc, "dg_basis_tables")
    return B, D, Mi


def kinetic_energy_noalloc(order: int, nelem: int, d_state: int, d_djac: int, d_ke: int, stream: int = 0):
    """Allocation-free kinetic energy on device pointers (dg_kinetic_energy_noalloc).

    For callers whose device memory is owned by their own allocator: the
    library allocates nothing; the result lands in the device double d_ke and
    the work is queued on `stream` without waiting for it."""
    lib = library()
    rc = lib.dg_kinetic_energy_noalloc(order, nelem, ctypes.c_void_p(d_state), ctypes.c_void_p(d_djac),
                                       ctypes.c_void_p(d_ke), ctypes.c_void_p(stream))
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())


def probe_bounded_wait(device: int, limit_cycles: int, arrive: bool) -> tuple[int, int]:
    """The failure-detection probe of the bounded device waits
    (dg_probe_bounded_wait): (return code, SM cycles the wait took); the code
    is DG_ERR_TIMEOUT when the wait gave up, 0 when the barrier completed."""
    lib = library()
    cyc = ctypes.c_longlong()
    rc = lib.dg_probe_bounded_wait(int(device), int(limit_cycles), 1 if arrive else 0, ctypes.byref(cyc))
    if rc not in (DG_OK, DG_ERR_TIMEOUT):
        raise DGError(rc, lib.dg_last_error(None).decode())
    return rc, cyc.value


# ---------------------------------------------------------------------------
# 2D quadrilaterals (dg2d_*)
# ---------------------------------------------------------------------------

def periodic_box_2d(n, x0=(0.0, 0.0), length=(1.0, 1.0), rotate_seed: int = 0) -> Mesh:
    """Periodic quadrilateral box from dg_mesh2d_periodic_box (a Mesh with dim 2)."""
    lib = library()
    n_arr = (ctypes.c_int * 2)(*[int(v) for v in n])
    x_arr = (ctypes.c_double * 2)(*[float(v) for v in x0])
    l_arr = (ctypes.c_double * 2)(*[float(v) for v in length])
    nn, ne, nf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = lib.dg_mesh2d_periodic_box(n_arr, x_arr, l_arr, ctypes.c_uint(rotate_seed), ctypes.byref(nn), None,
                                    ctypes.byref(ne), None, ctypes.byref(nf), None)
    if rc:
        raise DGError(rc, "dg_mesh2d_periodic_box: bad box")
    coords = np.zeros((nn.value, 2), np.float64)
    e2n = np.zeros((ne.value, 4), np.uint32)
    faces = np.zeros((nf.value, 8), np.uint32)
    rc = lib.dg_mesh2d_periodic_box(n_arr, x_arr, l_arr, ctypes.c_uint(rotate_seed), ctypes.byref(nn), _dptr(coords),
                                    ctypes.byref(ne), _uptr(e2n), ctypes.byref(nf), _uptr(faces))
    if rc:
        raise DGError(rc, "dg_mesh2d_periodic_box failed")
    return Mesh(coords, e2n, faces, 2, 1)


def _mesh2d_desc(mesh: Mesh, keep: list) -> _MeshDesc:
    c = np.ascontiguousarray(mesh.node_coords, np.float64)
    e = np.ascontiguousarray(mesh.elem_to_node_ids, np.uint32)
    f = np.ascontiguousarray(mesh.interior_faces, np.uint32)
    if c.ndim != 2 or c.shape[1] != 2 or e.ndim != 2 or e.shape[1] != 4 or f.ndim != 2 or f.shape[1] != 8:
        raise ValueError("the 2D path takes quadrilateral meshes (node_coords [n][2], elem_to_node_ids [ne][4], "
                         "interior_faces [nf][8])")
    keep += [c, e, f]
    return _MeshDesc(c.shape[0], _dptr(c), e.shape[0], _uptr(e), f.shape[0], _uptr(f), 0)


def write_solution_h5_2d(path, mesh: Mesh, order: int, Uc: np.ndarray, time: float = 0.0):
    """Uc[ne][nb][4] in the writer's data.h5 schema (dg2d_solution_write_h5)."""
    lib = library()
    keep = []
    md = _mesh2d_desc(mesh, keep)
    U = np.ascontiguousarray(Uc, np.float64)
    if U.size != mesh.nelem * (order + 1) ** 2 * 4:
        raise ValueError("Uc does not hold a 2D state of this mesh and order")
    rc = lib.dg2d_solution_write_h5(_path(path), ctypes.byref(md), int(order), _dptr(U), float(time))
    if rc:
        raise DGError(rc, lib.dg_last_error(None).decode())


class Case2D:
    """One 2D case (Solver<2> with LagrangeQuad) on the device: states
    Uc[ne][nb][4], nb = (p+1)^2, FP64."""

    def __init__(self, mesh: Mesh, order: int, flux: str = "LaxFriedrichs", gamma: float = 1.4,
                 gas_constant: float = 287.05, device: int = 0):
        self._lib = library()
        keep = []
        md = _mesh2d_desc(mesh, keep)
        cd = _CaseDesc(order, FLUX[flux], gamma, gas_constant, PRECISION["fp64"], device)
        h = ctypes.c_void_p()
        rc = self._lib.dg2d_create(ctypes.byref(cd), ctypes.byref(md), ctypes.byref(h))
        if rc:
            raise DGError(rc, self._lib.dg_last_error(None).decode())
        self._h = h
        self.order = order
        self.ne = mesh.nelem
        self.nb = self._lib.dg2d_num_basis(self._h)

    def _check(self, rc):
        if rc:
            raise DGError(rc, self._lib.dg2d_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dg2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, Uc: np.ndarray):
        U = np.ascontiguousarray(Uc, np.float64)
        if U.size != self.ne * self.nb * 4:
            raise ValueError("state size")
        self._check(self._lib.dg2d_set_state(self._h, _dptr(U)))

    def get_state(self) -> np.ndarray:
        U = np.zeros((self.ne, self.nb, 4))
        self._check(self._lib.dg2d_get_state(self._h, _dptr(U)))
        return U

    def residual(self) -> np.ndarray:
        R = np.zeros((self.ne, self.nb, 4))
        self._check(self._lib.dg2d_residual(self._h, _dptr(R)))
        return R

    def rk4(self, dt: float, nsteps: int):
        self._check(self._lib.dg2d_rk4_steps(self._h, dt, int(nsteps)))

    def rk4_timed(self, dt: float, nsteps: int) -> float:
        ms = ctypes.c_double()
        self._check(self._lib.dg2d_rk4_steps_timed(self._h, dt, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def fe(self, dt: float, nsteps: int):
        self._check(self._lib.dg2d_fe_steps(self._h, dt, int(nsteps)))

    def project_ic(self, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        U = np.zeros((self.ne, self.nb, 4))
        self._check(self._lib.dg2d_project_ic(self._h, IC2D[name], _dptr(d) if d.size else None, d.size, t,
                                              _dptr(U)))
        return U

    def l2_error(self, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        err = np.zeros(4)
        self._check(self._lib.dg2d_l2_error(self._h, IC2D[name], _dptr(d) if d.size else None, d.size, t,
                                            _dptr(err)))
        return err

    def status(self) -> int:
        f = ctypes.c_uint()
        self._lib.dg2d_status(self._h, ctypes.byref(f))
        return f.value
