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
        L.oracle_poly_vgl.restype = C.c_int
        L.oracle_poly_vgl.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
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
        if not self.h:
            raise ValueError("oracle: shell angular momentum outside 0..7")

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_basis_destroy(self.h)
            self.h = None


MAX_L = 7
NPOLY = 120


def poly_vgl(lmax, X, R, path="hpc"):
    """Cartesian monomials of degree <= lmax at X - R: (vgl[5][n], n).

    path "hpc" adds the 1e-20 shift after the products
    (org/qmckl_ao.org:6624-6914), "doc" to the displacement (6233-6364)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    R = np.ascontiguousarray(R, dtype=np.float64)
    out = np.zeros((5, NPOLY), dtype=np.float64)
    n = lib().oracle_poly_vgl(1 if path == "hpc" else 0, lmax, _p(X), _p(R), _p(out))
    if n < 0:
        raise ValueError("lmax outside 0..7")
    return out[:, :n], n


def monomial_powers(lmax):
    """(a, b, c) of every monomial of degree <= lmax in the reference's
    canonical order: l ascending, then a descending, then b descending
    (org/qmckl_ao.org:5928-5933)."""
    out = []
    for l in range(lmax + 1):
        for a in range(l, -1, -1):
            for b in range(l - a, -1, -1):
                out.append((a, b, l - a - b))
    return out


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


# ---------------------------------------------------------------- cusp-corrected MOs, MO Hessian
#
# numpy restatements of the reference's cusp adjustment and MO Hessian
# (org/qmckl_mo.org); the AO quantities they read come from the C restatement.

def ao_nucl_ang_mom(sysd):
    """(ao_nucl [A], ao_ang_mom [A]) as finalized by the reference
    (qmckl_finalize_basis, org/qmckl_ao.org:2965-3226): cartesian AOs shell by
    shell, (l+1)(l+2)/2 per shell."""
    nidx = np.asarray(sysd["nucleus_index"])
    nsh = np.asarray(sysd["nucleus_shell_num"])
    lsh = np.asarray(sysd["shell_ang_mom"])
    shell_nucl = np.empty(lsh.size, dtype=np.int64)
    for n in range(nidx.size):
        shell_nucl[nidx[n]:nidx[n] + nsh[n]] = n
    nucl, lval = [], []
    for s in range(lsh.size):
        k = (int(lsh[s]) + 1) * (int(lsh[s]) + 2) // 2
        nucl += [shell_nucl[s]] * k
        lval += [int(lsh[s])] * k
    return np.array(nucl, dtype=np.int64), np.array(lval, dtype=np.int32)


def en_distance(coord, nucl_coord):
    """[P][N] point-nucleus distances (qmckl_compute_en_distance,
    org/qmckl_electron.org:1357-1393, through qmckl_distance
    org/qmckl_distance.org:488-640: x = R - r, sqrt(x*x + y*y + z*z))."""
    c = np.asarray(coord, dtype=np.float64)               # [P][3]
    n = np.asarray(nucl_coord, dtype=np.float64)          # [3][N]
    x = n[0][None, :] - c[:, 0][:, None]
    y = n[1][None, :] - c[:, 1][:, None]
    z = n[2][None, :] - c[:, 2][:, None]
    return np.sqrt(x * x + y * y + z * z)


def mo_value_cusp(coefficient, ao_value_arr, ao_nucl, ao_l, en_dist, r_cusp, cusp_param):
    """qmckl_compute_mo_basis_mo_value_cusp_doc (org/qmckl_mo.org:2807-2860):
    the s AOs of a nucleus are left out at points closer than r_cusp (strictly),
    and the cubic c0 + c1 r + c2 r^2 + c3 r^3 of that nucleus is added where
    r <= r_cusp.  cusp_param [N][4][M]; returns [P][M]."""
    C = np.asarray(coefficient, dtype=np.float64)          # [M][A]
    rc = np.asarray(r_cusp, dtype=np.float64)
    skip = (ao_l[None, :] == 0) & (en_dist[:, ao_nucl] < rc[ao_nucl][None, :])
    mo = np.where(skip, 0.0, ao_value_arr) @ C.T
    for n in range(rc.size):
        inside = en_dist[:, n] <= rc[n]
        r = en_dist[inside, n][:, None]
        p = cusp_param[n]
        mo[inside] += p[0][None, :] + r * (p[1][None, :] + r * (p[2][None, :] + r * p[3][None, :]))
    return mo


def mo_vgl_cusp(coefficient, ao_vgl_arr, ao_nucl, ao_l, coord, nucl_coord, r_cusp, cusp_param):
    """qmckl_compute_mo_basis_mo_vgl_cusp_doc (org/qmckl_mo.org:3099-3185): AOs
    kept where r > r_cusp or l > 0; where r < r_cusp the cubic's value,
    gradient (c1/r + 2 c2 + 3 c3 r) (r - R) and Laplacian
    2 c1/r + 6 c2 + 12 c3 r are added.  Returns [P][5][M]."""
    C = np.asarray(coefficient, dtype=np.float64)
    rc = np.asarray(r_cusp, dtype=np.float64)
    pts = np.asarray(coord, dtype=np.float64)
    nuc = np.asarray(nucl_coord, dtype=np.float64)
    en = en_distance(pts, nuc)
    keep = (en[:, ao_nucl] > rc[ao_nucl][None, :]) | (ao_l[None, :] > 0)          # [P][A]
    mo = np.einsum("pck,ik->pci", np.where(keep[:, None, :], ao_vgl_arr, 0.0), C)
    for n in range(rc.size):
        inside = en[:, n] < rc[n]
        if not inside.any():
            continue
        r = en[inside, n][:, None]
        rv = pts[inside] - nuc[:, n][None, :]                                        # [p][3]
        p = cusp_param[n]
        mo[inside, 0] += p[0] + r * (p[1] + r * (p[2] + r * p[3]))
        c1 = p[1] / r + 2.0 * p[2] + r * 3.0 * p[3]
        for d in range(3):
            mo[inside, 1 + d] += rv[:, d][:, None] * c1
        mo[inside, 4] += 2.0 * p[1] / r + 6.0 * p[2] + 12.0 * p[3] * r
    return mo


def cusp_param(basis, sysd, r_cusp, precision=53):
    """Parameters of the cusp cubic of every (nucleus, MO), [N][4][M], as
    qmckl_set_mo_basis_r_cusp forms them (org/qmckl_mo.org:479-700): eta = the
    MO at the nucleus without the s AOs left out there (mo_value_cusp with
    zero parameters), phi / grad_phi / lap_phi = the nucleus's own s-AO part
    of the MO at distance r_cusp along z (value, z derivative, Laplacian);
    nuclei with charge < 0.1 keep zero parameters."""
    C = np.asarray(sysd["mo_coef"], dtype=np.float64)
    M = C.shape[0]
    nuc = np.asarray(sysd["nucl_coord"], dtype=np.float64)
    N = nuc.shape[1]
    rc = np.asarray(r_cusp, dtype=np.float64)
    Z = np.asarray(sysd["charge"], dtype=np.float64)
    ao_nucl, ao_l = ao_nucl_ang_mom(sysd)
    at = np.ascontiguousarray(nuc.T)                       # the nuclei as points
    eta = mo_value_cusp(C, ao_value(basis, at, nuc, precision), ao_nucl, ao_l, en_distance(at, nuc), rc,
                        np.zeros((N, 4, M)))               # [N][M]
    shifted = at.copy()
    shifted[:, 2] += rc
    av = ao_vgl(basis, shifted, nuc, precision)            # [N][5][A]
    out = np.zeros((N, 4, M))
    for n in range(N):
        s = (ao_nucl == n) & (ao_l == 0)
        phi = C[:, s] @ av[n, 0, s]
        gphi = C[:, s] @ av[n, 3, s]
        lphi = C[:, s] @ av[n, 4, s]
        if Z[n] < 0.1:
            continue
        R, z, e = rc[n], Z[n], eta[n]
        out[n, 0] = -(R * (2. * e * z - 6. * gphi) + lphi * R * R + 6. * phi) / (2. * R * z - 6.)
        out[n, 1] = (lphi * R * R * z - 6. * gphi * R * z + 6. * phi * z + 6. * e * z) / (2. * R * z - 6.)
        out[n, 2] = -(R * (-5. * gphi * z - 1.5 * lphi) + lphi * R * R * z + 3. * phi * z + 3. * e * z
                      + 6. * gphi) / (R * R * z - 3. * R)
        out[n, 3] = (R * (-2. * gphi * z - lphi) + 0.5 * lphi * R * R * z + phi * z + e * z + 3. * gphi) / \
            (R * R * R * z - 3. * R * R)
    return out


def mo_hessian(coefficient, ao_hessian_arr, ao_nucl=None, ao_l=None, coord=None, nucl_coord=None, r_cusp=None,
               cusp_param_arr=None):
    """MO Hessian [3][P][3][M] from ao_hessian [3][P][4][A]
    (qmckl_compute_mo_basis_mo_hessian_doc_f, org/qmckl_mo.org:2540-2575);
    with r_cusp, qmckl_compute_mo_basis_mo_hessian_cusp_doc_f (2629-2697):
    AOs kept where ao_hessian[jj][p][0][k] != 0 and (r > r_cusp or l > 0), and
    where r < r_cusp the cubic's Hessian
    c1 (delta/r - x x'/r^3) + 2 c2 delta + 3 c3 (delta r + x x'/r)."""
    C = np.asarray(coefficient, dtype=np.float64)
    H = np.asarray(ao_hessian_arr, dtype=np.float64)
    if r_cusp is None:
        return np.einsum("jpkq,iq->jpki", H[:, :, :3, :], C)
    rc = np.asarray(r_cusp, dtype=np.float64)
    pts = np.asarray(coord, dtype=np.float64)
    nuc = np.asarray(nucl_coord, dtype=np.float64)
    en = en_distance(pts, nuc)
    keep = ((en[:, ao_nucl] > rc[ao_nucl][None, :]) | (ao_l[None, :] > 0))[None, :, :] & (H[:, :, 0, :] != 0.0)
    out = np.einsum("jpkq,iq->jpki", np.where(keep[:, :, None, :], H[:, :, :3, :], 0.0), C)
    for n in range(rc.size):
        inside = en[:, n] < rc[n]
        if not inside.any():
            continue
        r = en[inside, n][:, None]
        rv = pts[inside] - nuc[:, n][None, :]
        p = cusp_param_arr[n]
        for jj in range(3):
            for kk in range(3):
                t = -p[1] * rv[:, kk][:, None] * rv[:, jj][:, None] / r ** 3 + \
                    p[3] * 3 * rv[:, kk][:, None] * rv[:, jj][:, None] / r
                if kk == jj:
                    t = t + p[1] / r + p[2] * 2 + p[3] * 3 * r
                out[jj, inside, kk] += t
    return out
