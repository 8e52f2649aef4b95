"""Oracle restatements of the cusp-corrected MOs and of the MO Hessian
(test infrastructure), pinned by the conditions that define them.

* The cusp cubic of nucleus A replaces A's s AOs inside r_cusp; its four
  parameters (org/qmckl_mo.org:479-700) are fixed by Kato's cusp condition
  at the nucleus, c1 = -Z (eta + c0), and by continuity of the value, the
  radial derivative and the Laplacian at r_cusp.  The tests check both on the
  restated mo_vgl_cusp: across the sphere r = r_cusp (in random directions)
  all five components are continuous.
* The MO Hessian is pinned like the reference pins it
  (org/qmckl_mo.org:3887-3985): a 9-point finite difference, over the nuclear
  coordinates, of the MO gradient rows of mo_vgl (step 1e-5, |diff| < 1e-8),
  on CHBrClF; the cusp-corrected Hessian against central differences of the
  cusp-corrected gradient over the point coordinates.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from qmckl_b200 import gen

STENCIL = np.array([1 / 280, -4 / 105, 1 / 5, -4 / 5, 0.0, 4 / 5, -1 / 5, 4 / 105, -1 / 280])


def cusp_system():
    d = gen.config(0, walk_num=1)
    rc = np.where(np.asarray(d["charge"]) > 1.5, 0.2, 0.5)
    return d, rc


def near_nuclei(d, rc, per=6, seed=3):
    """Points inside the cusp spheres (0.05 .. 0.95 r_cusp) and a few outside."""
    rng = np.random.default_rng(seed)
    nuc = np.asarray(d["nucl_coord"]).T
    pts = []
    for n in range(nuc.shape[0]):
        u = rng.standard_normal((per, 3))
        u /= np.linalg.norm(u, axis=1)[:, None]
        r = rc[n] * rng.uniform(0.05, 0.95, per)
        pts.append(nuc[n] + u * r[:, None])
    pts.append(gen.points(d)[:20])
    return np.concatenate(pts)


def test_cusp_parameters_satisfy_kato_and_continuity():
    d, rc = cusp_system()
    basis = O.Basis(d)
    prm = O.cusp_param(basis, d, rc)                      # [N][4][M]
    C = d["mo_coef"]
    N, M = prm.shape[0], prm.shape[2]
    nuc = np.asarray(d["nucl_coord"])
    an, al = O.ao_nucl_ang_mom(d)
    # Kato's condition at the nucleus
    at = np.ascontiguousarray(nuc.T)
    eta = O.mo_value_cusp(C, O.ao_value(basis, at, nuc), an, al, O.en_distance(at, nuc), rc, np.zeros((N, 4, M)))
    Z = np.asarray(d["charge"])
    for n in range(N):
        lhs, rhs = prm[n, 1], -Z[n] * (eta[n] + prm[n, 0])
        assert np.abs(lhs - rhs).max() <= 1e-10 * max(1.0, np.abs(lhs).max())
    # continuity of value, gradient and Laplacian across r = r_cusp
    rng = np.random.default_rng(9)
    for n in range(N):
        u = rng.standard_normal((4, 3))
        u /= np.linalg.norm(u, axis=1)[:, None]
        for eps in (-1e-9, 1e-9):
            pts = at[n] + u * rc[n] * (1.0 + eps)
            v = O.mo_vgl_cusp(C, O.ao_vgl(basis, pts, nuc, path="doc"), an, al, pts, nuc, rc, prm)
            if eps < 0:
                inner = v
            else:
                outer = v
        scale = np.abs(outer).max(axis=(0, 2))            # per component
        jump = np.abs(inner - outer).max(axis=(0, 2))
        assert (jump <= 1e-6 * scale).all(), (n, jump / scale)


def test_cusp_parameters_zero_for_dummy_atoms():
    d, rc = cusp_system()
    d = dict(d)
    ch = np.array(d["charge"], dtype=np.float64)
    ch[0] = 0.0
    d["charge"] = ch
    prm = O.cusp_param(O.Basis(d), d, rc)
    assert not prm[0].any()
    assert prm[1:].any()


def test_mo_hessian_matches_nuclear_finite_difference(chbrclf):
    basis = O.Basis(chbrclf)
    pts = chbrclf["elec_coord"][0]
    nucl = np.array(chbrclf["nucl_coord"], dtype=np.float64)
    C = chbrclf["mo_coef"]
    N, P, M = nucl.shape[1], pts.shape[0], C.shape[0]
    mh = O.mo_hessian(C, O.ao_hessian(basis, pts, nucl))  # [3][P][3][M]
    fd = np.zeros((3, P, 3, M))
    dx = 1.0e-5
    for a in range(N):
        for k in range(3):
            for m in range(-4, 5):
                if m == 0:
                    continue
                t = nucl.copy()
                t[k, a] += m * dx
                mo = O.mo_vgl(C, O.ao_vgl(basis, pts, t, path="doc"))
                fd[k] -= STENCIL[m + 4] * mo[:, 1:4, :] / dx
    assert np.abs(fd - mh).max() < 1e-8


def test_cusp_mo_hessian_matches_point_finite_difference():
    d, rc = cusp_system()
    basis = O.Basis(d)
    prm = O.cusp_param(basis, d, rc)
    C = d["mo_coef"]
    nuc = np.asarray(d["nucl_coord"])
    an, al = O.ao_nucl_ang_mom(d)
    pts = near_nuclei(d, rc)
    mh = O.mo_hessian(C, O.ao_hessian(basis, pts, nuc), an, al, pts, nuc, rc, prm)
    h = 1.0e-5
    fd = np.zeros_like(mh)
    for jj in range(3):
        for m in range(-4, 5):
            if m == 0:
                continue
            q = pts.copy()
            q[:, jj] += m * h
            v = O.mo_vgl_cusp(C, O.ao_vgl(basis, q, nuc, path="doc"), an, al, q, nuc, rc, prm)
            fd[jj] += STENCIL[m + 4] * v[:, 1:4, :] / h
    scale = np.abs(mh).max(axis=(0, 2, 3))                # per point
    err = np.abs(fd - mh).max(axis=(0, 2, 3))
    assert (err <= 1e-6 * np.maximum(scale, 1.0)).all(), (err / np.maximum(scale, 1.0)).max()
