"""ctypes face of oracle/_ref/libqmckl_ref.so: the reference's own C HPC
kernels (qmckl_finalize_basis, qmckl_compute_ao_vgl_hpc_gaussian,
qmckl_compute_ao_value_hpc_gaussian, qmckl_compute_mo_basis_mo_vgl_hpc,
qmckl_compute_mo_basis_mo_value_hpc), compiled from the reference's sources
by oracle/build_ref.py.  Test infrastructure only: the checker of the oracle
and the CPU baseline of bench.py.  The library exists where the reference's
sources were present at build time; available() says whether it does."""
import ctypes as C
import os

import numpy as np

from . import build_ref as _build

_lib = None


class _SystemIn(C.Structure):
    _fields_ = [("nucl_num", C.c_int64), ("shell_num", C.c_int64), ("prim_num", C.c_int64), ("ao_num", C.c_int64),
                ("nucl_coord", C.c_void_p), ("nucleus_index", C.c_void_p), ("nucleus_shell_num", C.c_void_p),
                ("shell_ang_mom", C.c_void_p), ("shell_prim_num", C.c_void_p), ("shell_prim_index", C.c_void_p),
                ("shell_factor", C.c_void_p), ("exponent", C.c_void_p), ("coefficient", C.c_void_p),
                ("prim_factor", C.c_void_p), ("ao_factor", C.c_void_p), ("precision", C.c_int32),
                ("num_threads", C.c_int32)]


def available():
    return os.path.exists(_build.LIB)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/libqmckl_ref.so is not built (python -m oracle.build_ref)")
        L = C.CDLL(_build.LIB)
        L.ref_system_create.restype = C.c_void_p
        L.ref_system_create.argtypes = [C.POINTER(_SystemIn)]
        L.ref_system_destroy.argtypes = [C.c_void_p]
        L.ref_system_set.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
        for f in ("ref_ao_vgl", "ref_ao_value"):
            getattr(L, f).restype = C.c_int32
            getattr(L, f).argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        for f in ("ref_mo_vgl", "ref_mo_value"):
            getattr(L, f).restype = C.c_int32
            getattr(L, f).argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class RefSystem:
    """A system dict (qmckl_b200.gen) finalized by the reference's own code."""

    def __init__(self, sysd, precision=53, num_threads=1):
        k = {n: np.ascontiguousarray(sysd[n], dtype=t) for n, t in (
            ("nucl_coord", np.float64), ("nucleus_index", np.int64), ("nucleus_shell_num", np.int64),
            ("shell_ang_mom", np.int32), ("shell_prim_num", np.int64), ("shell_prim_index", np.int64),
            ("shell_factor", np.float64), ("exponent", np.float64), ("coefficient", np.float64),
            ("prim_factor", np.float64), ("ao_factor", np.float64))}
        self._keep = k
        self.ao_num = k["ao_factor"].size
        self.mo_num = int(sysd["mo_coef"].shape[0])
        self.coef_t = np.ascontiguousarray(np.asarray(sysd["mo_coef"], dtype=np.float64).T)   # [ao][mo]
        si = _SystemIn(k["nucleus_index"].size, k["shell_ang_mom"].size, k["exponent"].size, self.ao_num,
                       *(_p(k[n]) for n in ("nucl_coord", "nucleus_index", "nucleus_shell_num", "shell_ang_mom",
                                            "shell_prim_num", "shell_prim_index", "shell_factor", "exponent",
                                            "coefficient", "prim_factor", "ao_factor")),
                       precision, num_threads)
        self.h = lib().ref_system_create(C.byref(si))
        if not self.h:
            raise RuntimeError("the reference's qmckl_finalize_basis failed")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.ref_system_destroy(self.h)
            self.h = None

    def set(self, precision=0, nthreads=0):
        lib().ref_system_set(self.h, precision, nthreads)

    def _coords(self, pts):
        return np.ascontiguousarray(np.asarray(pts, dtype=np.float64).T)   # [3][P]

    def ao_vgl(self, pts, nthreads=0):
        self.set(0, nthreads)
        c = self._coords(pts)
        out = np.empty((c.shape[1], 5, self.ao_num))
        rc = lib().ref_ao_vgl(self.h, c.shape[1], _p(c), _p(out))
        if rc != 0:
            raise RuntimeError(f"qmckl_compute_ao_vgl_hpc_gaussian returned {rc}")
        return out

    def ao_value(self, pts, nthreads=0):
        self.set(0, nthreads)
        c = self._coords(pts)
        out = np.empty((c.shape[1], self.ao_num))
        rc = lib().ref_ao_value(self.h, c.shape[1], _p(c), _p(out))
        if rc != 0:
            raise RuntimeError(f"qmckl_compute_ao_value_hpc_gaussian returned {rc}")
        return out

    def mo_vgl(self, pts, nthreads=0, ao=None):
        ao = self.ao_vgl(pts, nthreads) if ao is None else np.ascontiguousarray(ao)
        self.set(0, nthreads)
        out = np.empty((ao.shape[0], 5, self.mo_num))
        rc = lib().ref_mo_vgl(self.h, self.mo_num, _p(self.coef_t), ao.shape[0], _p(ao), _p(out))
        if rc != 0:
            raise RuntimeError(f"qmckl_compute_mo_basis_mo_vgl_hpc returned {rc}")
        return out

    def mo_value(self, pts, nthreads=0):
        ao = self.ao_value(pts, nthreads)
        self.set(0, nthreads)
        out = np.empty((ao.shape[0], self.mo_num))
        rc = lib().ref_mo_value(self.h, self.mo_num, _p(self.coef_t), ao.shape[0], _p(ao), _p(out))
        if rc != 0:
            raise RuntimeError(f"qmckl_compute_mo_basis_mo_value_hpc returned {rc}")
        return out
