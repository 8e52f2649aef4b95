"""ctypes face of the CPU oracle (oracle.c).  Test infrastructure only."""
import ctypes as C
import os

import numpy as np

from . import build as _build

_lib = None
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


class _BasisIn(C.Structure):
    _fields_ = [("nucl_num", C.c_int64), ("shell_num", C.c_int64), ("prim_num", C.c_int64),
                ("ao_num", C.c_int64),
                ("nucleus_index", C.c_void_p), ("nucleus_shell_num", C.c_void_p),
                ("shell_ang_mom", C.c_void_p), ("shell_prim_num", C.c_void_p),
                ("shell_prim_index", C.c_void_p), ("shell_factor", C.c_void_p),
                ("exponent", C.c_void_p), ("coefficient", C.c_void_p),
                ("prim_factor", C.c_void_p), ("ao_factor", C.c_void_p)]


def lib():
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            path = _build.build()
        L = C.CDLL(path)
        L.oracle_basis_create.restype = C.c_void_p
        L.oracle_basis_create.argtypes = [C.POINTER(_BasisIn)]
        L.oracle_basis_destroy.argtypes = [C.c_void_p]
        L.oracle_cutoff.restype = C.c_double
        L.oracle_cutoff.argtypes = [C.c_int32]
        L.oracle_nucleus_range.restype = C.c_double
        L.oracle_nucleus_range.argtypes = [C.c_void_p, C.c_int64]
        L.oracle_prim_per_nucleus.restype = C.c_int64
        L.oracle_prim_per_nucleus.argtypes = [C.c_void_p, C.c_int64]
        for f in ("oracle_ao_vgl_hpc", "oracle_ao_value_hpc"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
        for f in ("oracle_primitive_vgl", "oracle_shell_vgl_doc", "oracle_ao_vgl_doc"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        for f in ("oracle_shell_hessian_doc", "oracle_ao_hessian_doc"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_mo_vgl_adjoint.argtypes = [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_forces.argtypes = [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        for f in ("oracle_mo_vgl", "oracle_mo_value"):
            getattr(L, f).argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Basis:
    """Finalized basis tables for a system dict (see qmckl_b200.gen)."""

    def __init__(self, sysd):
        self._keep = {k: np.ascontiguousarray(sysd[k], dtype=t) for k, t in (
            ("nucleus_index", np.int64), ("nucleus_shell_num", np.int64), ("shell_ang_mom", np.int32),
            ("shell_prim_num", np.int64), ("shell_prim_index", np.int64), ("shell_factor", np.float64),
            ("exponent", np.float64), ("coefficient", np.float64), ("prim_factor", np.float64),
            ("ao_factor", np.float64))}
        k = self._keep
        self.nucl_num = k["nucleus_index"].size
        self.shell_num = k["shell_ang_mom"].size
        self.prim_num = k["exponent"].size
        self.ao_num = k["ao_factor"].size
        bi = _BasisIn(self.nucl_num, self.shell_num, self.prim_num, self.ao_num,
                      *(_p(k[n]) for n in ("nucleus_index", "nucleus_shell_num", "shell_ang_mom",
                                            "shell_prim_num", "shell_prim_index", "shell_factor",
                                            "exponent", "coefficient", "prim_factor", "ao_factor")))
        self.h = lib().oracle_basis_create(C.byref(bi))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_basis_destroy(self.h)
            self.h = None


def _coords(coord, nucl_coord):
    """coord: [P,3] (x,y,z per point) -> [3][P] column blocks; nucl_coord [3][N]."""
    c = np.ascontiguousarray(np.asarray(coord, dtype=np.float64).T)
    n = np.ascontiguousarray(np.asarray(nucl_coord, dtype=np.float64))
    return c, n


def ao_vgl(basis, coord, nucl_coord, precision=53, path="hpc", nthreads=0):
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    out = np.empty((P, 5, basis.ao_num), dtype=np.float64)
    if path == "hpc":
        lib().oracle_ao_vgl_hpc(basis.h, precision, P, _p(c), _p(n), _p(out), nthreads)
    else:
        lib().oracle_ao_vgl_doc(basis.h, precision, P, _p(c), _p(n), _p(out))
    return out


def ao_value(basis, coord, nucl_coord, precision=53, nthreads=0):
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    out = np.empty((P, basis.ao_num), dtype=np.float64)
    lib().oracle_ao_value_hpc(basis.h, precision, P, _p(c), _p(n), _p(out), nthreads)
    return out


def primitive_vgl(basis, coord, nucl_coord, precision=53):
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    out = np.empty((P, 5, basis.prim_num), dtype=np.float64)
    lib().oracle_primitive_vgl(basis.h, precision, P, _p(c), _p(n), _p(out))
    return out


def shell_vgl(basis, coord, nucl_coord, precision=53):
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    out = np.empty((P, 5, basis.shell_num), dtype=np.float64)
    lib().oracle_shell_vgl_doc(basis.h, precision, P, _p(c), _p(n), _p(out))
    return out


def mo_vgl(coefficient, ao_vgl_arr, nthreads=0):
    """coefficient: [mo][ao] (the qmckl_set_mo_basis_coefficient layout)."""
    ct = np.ascontiguousarray(np.asarray(coefficient, dtype=np.float64).T)   # [ao][mo]
    a = np.ascontiguousarray(ao_vgl_arr, dtype=np.float64)
    P, _, A = a.shape
    M = ct.shape[1]
    out = np.empty((P, 5, M), dtype=np.float64)
    lib().oracle_mo_vgl(A, M, P, _p(ct), _p(a), _p(out), nthreads)
    return out


def mo_value(coefficient, ao_value_arr, nthreads=0):
    ct = np.ascontiguousarray(np.asarray(coefficient, dtype=np.float64).T)
    a = np.ascontiguousarray(ao_value_arr, dtype=np.float64)
    P, A = a.shape
    M = ct.shape[1]
    out = np.empty((P, M), dtype=np.float64)
    lib().oracle_mo_value(A, M, P, _p(ct), _p(a), _p(out), nthreads)
    return out


def shell_hessian(basis, coord, nucl_coord, precision=53):
    """[P][3][4][shell] (qmckl_get_ao_basis_shell_hessian layout)."""
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    out = np.empty((P, 3, 4, basis.shell_num), dtype=np.float64)
    lib().oracle_shell_hessian_doc(basis.h, precision, P, _p(c), _p(n), _p(out))
    return out


def ao_hessian(basis, coord, nucl_coord, precision=53):
    """[3][P][4][ao] (qmckl_get_ao_basis_ao_hessian layout)."""
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    out = np.empty((3, P, 4, basis.ao_num), dtype=np.float64)
    lib().oracle_ao_hessian_doc(basis.h, precision, P, _p(c), _p(n), _p(out))
    return out


def mo_vgl_adjoint(basis, coord, nucl_coord, coefficient, weight, precision=53):
    """Gradient of sum(weight * mo_vgl): (grad_coef [mo][ao], grad_nucl [nucl][3], grad_coord [P][3])."""
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    coef = np.ascontiguousarray(coefficient, dtype=np.float64)
    M = coef.shape[0]
    w = np.ascontiguousarray(weight, dtype=np.float64).reshape(P, 5, M)
    gc = np.empty((M, basis.ao_num))
    gn = np.empty((basis.nucl_num, 3))
    gr = np.empty((3, P))
    lib().oracle_mo_vgl_adjoint(basis.h, precision, P, _p(c), _p(n), M, _p(coef), _p(w), _p(gc), _p(gn), _p(gr))
    return gc, gn, np.ascontiguousarray(gr.T)


def forces(basis, coord, nucl_coord, coefficient, precision=53):
    """(forces_ao_value [N][P][3][A], forces_mo_value [N][P][3][M], forces_mo_g [N][3][P][3][M],
    forces_mo_l [N][3][P][M])."""
    c, n = _coords(coord, nucl_coord)
    P = c.shape[1]
    coef = np.ascontiguousarray(coefficient, dtype=np.float64)
    M, A, N = coef.shape[0], basis.ao_num, basis.nucl_num
    fao = np.empty((N, P, 3, A))
    fmv = np.empty((N, P, 3, M))
    fmg = np.empty((N, 3, P, 3, M))
    fml = np.empty((N, 3, P, M))
    lib().oracle_forces(basis.h, precision, P, _p(c), _p(n), M, _p(coef), _p(fao), _p(fmv), _p(fmg), _p(fml))
    return fao, fmv, fmg, fml


def cutoff(precision=53):
    return lib().oracle_cutoff(precision)
