"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
CPU-baseline leg of bench.py, as the checker.  The product never uses it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

FLUX = {"LaxFriedrichs": 0, "HLLC": 1}
IC = {"Uniform": 0, "IsentropicVortex": 1, "Sphere": 2, "IsentropicVortexXY": 3, "TaylorGreen": 4}

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def library() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = ctypes.CDLL(LIB_PATH)
    d, i, v = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), ctypes.c_void_p
    sig = {
        "orc_hex_quadrature_order": (ctypes.c_int, [ctypes.c_int]),
        "orc_quad_quadrature_order": (ctypes.c_int, [ctypes.c_int]),
        "orc_segment_quadrature_order": (ctypes.c_int, [ctypes.c_int]),
        "orc_num_quadrature_points_1d": (ctypes.c_int, [ctypes.c_int]),
        "orc_gauss_legendre_1d": (None, [ctypes.c_int, d, d]),
        "orc_equidistant_nodes": (None, [ctypes.c_double, ctypes.c_double, ctypes.c_int, d]),
        "orc_lagrange_hex_val": (None, [ctypes.c_int, ctypes.c_int, d, d]),
        "orc_lagrange_hex_grad": (None, [ctypes.c_int, ctypes.c_int, d, d]),
        "orc_face_pts_order": (None, [ctypes.c_int, ctypes.c_int, i]),
        "orc_points_on_face": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_int, d, d]),
        "orc_local_nodes_on_face": (None, [ctypes.c_int, ctypes.c_int, i]),
        "orc_pressure": (ctypes.c_double, [ctypes.c_double, d]),
        "orc_maxwavespeed": (ctypes.c_double, [ctypes.c_double, d]),
        "orc_conv_flux": (None, [ctypes.c_double, d, d]),
        "orc_num_flux": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, d, d, d, d]),
        "orc_ic_eval": (None, [ctypes.c_int, ctypes.c_int, d, ctypes.c_double, ctypes.c_double, d,
                               ctypes.c_double, d]),
        "orc_create": (v, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, d,
                           ctypes.c_int, i, ctypes.c_int, i]),
        "orc_destroy": (None, [v]),
        "orc_nb": (ctypes.c_int, [v]),
        "orc_nqf": (ctypes.c_int, [v]),
        "orc_set_ic": (None, [v, ctypes.c_int, ctypes.c_int, d]),
        "orc_project_ic": (None, [v, ctypes.c_double, d]),
        "orc_residual": (None, [v, d, d]),
        "orc_rk4_steps": (None, [v, d, ctypes.c_double, ctypes.c_int]),
        "orc_fe_steps": (None, [v, d, ctypes.c_double, ctypes.c_int]),
        "orc_l2_error": (None, [v, d, ctypes.c_double, d]),
        "orc_total_volume": (ctypes.c_double, [v]),
        "orc_face_normals": (None, [v, d]),
        "orc_face_quad_idx": (None, [v, i, i]),
        "orc_face_points_phys": (None, [v, ctypes.c_int, ctypes.c_int, d]),
        "orc_flux_failures": (ctypes.c_long, [v]),
        "orc_set_threads": (None, [ctypes.c_int]),
        "orc_get_threads": (ctypes.c_int, []),
        "orc_inv_lu": (None, [ctypes.c_int, d, d]),
        "orc2_create": (v, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, d,
                            ctypes.c_int, i, ctypes.c_int, i]),
        "orc2_destroy": (None, [v]),
        "orc2_nb": (ctypes.c_int, [v]),
        "orc2_nqf": (ctypes.c_int, [v]),
        "orc2_set_ic": (None, [v, ctypes.c_int, ctypes.c_int, d]),
        "orc2_project_ic": (None, [v, ctypes.c_double, d]),
        "orc2_residual": (None, [v, d, d]),
        "orc2_rk4_steps": (None, [v, d, ctypes.c_double, ctypes.c_int]),
        "orc2_fe_steps": (None, [v, d, ctypes.c_double, ctypes.c_int]),
        "orc2_l2_error": (None, [v, d, ctypes.c_double, d]),
        "orc2_total_volume": (ctypes.c_double, [v]),
        "orc2_flux_failures": (ctypes.c_long, [v]),
        "orc2_face_normals": (None, [v, d]),
        "orc2_points_on_face": (None, [ctypes.c_int, ctypes.c_int, ctypes.c_int, d, d]),
        "orc2_face_pts_order": (None, [ctypes.c_int, ctypes.c_int, i]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def gauss_legendre(qorder: int):
    lib = library()
    n = lib.orc_num_quadrature_points_1d(qorder)
    x, w = np.zeros(n), np.zeros(n)
    lib.orc_gauss_legendre_1d(qorder, _d(x), _d(w))
    return x, w


def face_pts_order(orient: int, npts: int) -> np.ndarray:
    out = np.zeros(npts, np.int32)
    library().orc_face_pts_order(orient, npts, _i(out))
    return out


def num_flux(kind: str, gamma: float, UL, UR, N):
    UL, UR, N = (np.ascontiguousarray(a, np.float64) for a in (UL, UR, N))
    F = np.zeros(5)
    rc = library().orc_num_flux(FLUX[kind], gamma, _d(UL), _d(UR), _d(N), _d(F))
    return F, rc


def conv_flux(gamma: float, U) -> np.ndarray:
    U = np.ascontiguousarray(U, np.float64)
    F = np.zeros(15)
    library().orc_conv_flux(gamma, _d(U), _d(F))
    return F


class OracleCase:
    """The reference's dense algorithm on one mesh (CPU, OpenMP)."""

    def __init__(self, coords, e2n, iface_data, order: int, flux: str = "LaxFriedrichs", gamma: float = 1.4,
                 gas_constant: float = 287.05):
        lib = library()
        self._coords = np.ascontiguousarray(coords, np.float64)
        self._e2n = np.ascontiguousarray(e2n, np.int32)
        self._ifd = np.ascontiguousarray(iface_data, np.int32)
        self.ne = self._e2n.shape[0]
        self.order = order
        self._h = lib.orc_create(order, FLUX[flux], gamma, gas_constant, self._coords.shape[0], _d(self._coords),
                                 self.ne, _i(self._e2n), self._ifd.shape[0], _i(self._ifd))
        if not self._h:
            raise ValueError("orc_create failed")
        self.nb = lib.orc_nb(self._h)
        self.nqf = lib.orc_nqf(self._h)

    @classmethod
    def from_mesh(cls, mesh, order, **kw):
        return cls(mesh.node_coords, mesh.elem_to_node_ids.astype(np.int32), mesh.iface_data(), order, **kw)

    def close(self):
        if getattr(self, "_h", None):
            library().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def project_ic(self, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        lib = library()
        lib.orc_set_ic(self._h, IC[name], d.size, _d(d) if d.size else None)
        U = np.zeros((self.ne, self.nb, 5))
        lib.orc_project_ic(self._h, t, _d(U))
        return U

    def residual(self, U) -> np.ndarray:
        U = np.ascontiguousarray(U, np.float64)
        R = np.zeros_like(U)
        library().orc_residual(self._h, _d(U), _d(R))
        return R

    def rk4(self, U, dt: float, nsteps: int) -> np.ndarray:
        U = np.array(U, np.float64, copy=True, order="C")
        library().orc_rk4_steps(self._h, _d(U), dt, nsteps)
        return U

    def fe(self, U, dt: float, nsteps: int) -> np.ndarray:
        U = np.array(U, np.float64, copy=True, order="C")
        library().orc_fe_steps(self._h, _d(U), dt, nsteps)
        return U

    def l2_error(self, U, name: str, data=(), t: float = 0.0) -> np.ndarray:
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        lib = library()
        lib.orc_set_ic(self._h, IC[name], d.size, _d(d) if d.size else None)
        U = np.ascontiguousarray(U, np.float64)
        err = np.zeros(5)
        lib.orc_l2_error(self._h, _d(U), t, _d(err))
        return err

    def total_volume(self) -> float:
        return library().orc_total_volume(self._h)

    def face_normals(self) -> np.ndarray:
        N = np.zeros((self._ifd.shape[0], self.nqf, 3))
        library().orc_face_normals(self._h, _d(N))
        return N

    def face_points(self, elem: int, face: int) -> np.ndarray:
        X = np.zeros((self.nqf, 3))
        library().orc_face_points_phys(self._h, elem, face, _d(X))
        return X

    def quad_idx(self):
        L = np.zeros((self._ifd.shape[0], self.nqf), np.int32)
        R = np.zeros_like(L)
        library().orc_face_quad_idx(self._h, _i(L), _i(R))
        return L, R

    def flux_failures(self) -> int:
        return library().orc_flux_failures(self._h)


# 2D initial conditions: the reference's 2D vortex, or the 3D families at (x, y, 0)
IC2 = {"Uniform": 0, "IsentropicVortex": 5, "IsentropicVortexXY": 3}


class OracleCase2D:
    """The reference's dense 2D algorithm (Solver<2>, LagrangeQuad) on one
    quadrilateral mesh (CPU, OpenMP); states Uc[ne][nb][4]."""

    def __init__(self, coords, e2n, iface_data, order: int, flux: str = "LaxFriedrichs", gamma: float = 1.4,
                 gas_constant: float = 287.05):
        lib = library()
        self._coords = np.ascontiguousarray(coords, np.float64)
        self._e2n = np.ascontiguousarray(e2n, np.int32)
        self._ifd = np.ascontiguousarray(iface_data, np.int32)
        self.ne = self._e2n.shape[0]
        self.order = order
        self._h = lib.orc2_create(order, FLUX[flux], gamma, gas_constant, self._coords.shape[0], _d(self._coords),
                                  self.ne, _i(self._e2n), self._ifd.shape[0], _i(self._ifd))
        if not self._h:
            raise ValueError("orc2_create failed")
        self.nb = lib.orc2_nb(self._h)
        self.nqf = lib.orc2_nqf(self._h)

    @classmethod
    def from_mesh(cls, mesh, order, **kw):
        """From a 2D mesh object with node_coords [n][2], elem_to_node_ids
        [ne][4] and interior_faces [nf][8] rows."""
        f = np.asarray(mesh.interior_faces)
        return cls(mesh.node_coords, np.asarray(mesh.elem_to_node_ids).astype(np.int32),
                   f[:, [1, 2, 3, 5, 6, 7]].astype(np.int32), order, **kw)

    def close(self):
        if getattr(self, "_h", None):
            library().orc2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ic(self, name, data):
        d = np.ascontiguousarray(np.asarray(data, np.float64).reshape(-1))
        library().orc2_set_ic(self._h, IC2[name], d.size, _d(d) if d.size else None)

    def project_ic(self, name: str, data=(), t: float = 0.0) -> np.ndarray:
        self._ic(name, data)
        U = np.zeros((self.ne, self.nb, 4))
        library().orc2_project_ic(self._h, t, _d(U))
        return U

    def residual(self, U) -> np.ndarray:
        U = np.ascontiguousarray(U, np.float64)
        R = np.zeros_like(U)
        library().orc2_residual(self._h, _d(U), _d(R))
        return R

    def rk4(self, U, dt: float, nsteps: int) -> np.ndarray:
        U = np.array(U, np.float64, copy=True, order="C")
        library().orc2_rk4_steps(self._h, _d(U), dt, nsteps)
        return U

    def fe(self, U, dt: float, nsteps: int) -> np.ndarray:
        U = np.array(U, np.float64, copy=True, order="C")
        library().orc2_fe_steps(self._h, _d(U), dt, nsteps)
        return U

    def l2_error(self, U, name: str, data=(), t: float = 0.0) -> np.ndarray:
        self._ic(name, data)
        U = np.ascontiguousarray(U, np.float64)
        err = np.zeros(4)
        library().orc2_l2_error(self._h, _d(U), t, _d(err))
        return err

    def total_volume(self) -> float:
        return library().orc2_total_volume(self._h)

    def face_normals(self) -> np.ndarray:
        N = np.zeros((self._ifd.shape[0], self.nqf, 2))
        library().orc2_face_normals(self._h, _d(N))
        return N

    def flux_failures(self) -> int:
        return library().orc2_flux_failures(self._h)
