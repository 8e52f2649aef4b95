"""Oracle derivatives (test infrastructure) pinned the way the reference pins them.

* AO Hessian: the reference's own test (org/qmckl_ao.org:9806-9858) compares
  qmckl_get_ao_basis_ao_hessian with a 9-point finite difference, over the
  nuclear coordinates, of the gradient and Laplacian rows of ao_vgl
  (step 1e-5, |diff| < 1e-8).  Same test on the oracle, on CHBrClF.
* Orbital forces / adjoint: central finite differences of
  L = sum W * mo_vgl over the nuclear coordinates, the reference's
  qmckl_finite_difference_deriv_n stencil (org/qmckl_forces.org:424-546).
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from qmckl_b200 import gen

STENCIL = np.array([1 / 280, -4 / 105, 1 / 5, -4 / 5, 0.0, 4 / 5, -1 / 5, 4 / 105, -1 / 280])


@pytest.fixture(scope="module")
def basis(chbrclf):
    return O.Basis(chbrclf)


def test_ao_hessian_matches_nuclear_finite_difference(chbrclf, basis):
    pts = chbrclf["elec_coord"][0]
    nucl = np.array(chbrclf["nucl_coord"], dtype=np.float64)     # [3][N]
    N = nucl.shape[1]
    hess = O.ao_hessian(basis, pts, nucl)                          # [3][P][4][A]
    P, A = pts.shape[0], basis.ao_num
    fd = np.zeros((3, P, 4, A))
    dx = 1.0e-5
    # d/dR_a of an AO centred on a is -d/dr; summing the stencil over every
    # nucleus a collects each AO exactly once
    for a in range(N):
        for k in range(3):
            for m in range(-4, 5):
                if m == 0:
                    continue
                t = nucl.copy()
                t[k, a] += m * dx
                v = O.ao_vgl(basis, pts, t, path="doc")            # [P][5][A]
                fd[k] -= STENCIL[m + 4] * v[:, 1:5, :] / dx
    assert np.abs(fd - hess).max() < 1.0e-8


def test_shell_hessian_symmetric_and_traced(chbrclf, basis):
    pts = chbrclf["elec_coord"][0]
    sh = O.shell_hessian(basis, pts, chbrclf["nucl_coord"])        # [P][3][4][S]
    assert np.abs(sh[:, :, :3, :] - np.swapaxes(sh[:, :, :3, :], 1, 2)).max() < 1e-13
    # trace of the Hessian is the Laplacian of shell_vgl
    sv = O.shell_vgl(basis, pts, chbrclf["nucl_coord"])
    tr = sh[:, 0, 0, :] + sh[:, 1, 1, :] + sh[:, 2, 2, :]
    scale = np.abs(sv[:, 4, :]).max()
    assert np.abs(tr - sv[:, 4, :]).max() < 1e-12 * scale


def _loss(basis, coef, w, pts, nucl):
    av = O.ao_vgl(basis, pts, nucl, path="doc")
    return float((w * O.mo_vgl(coef, av)).sum())


def test_adjoint_matches_finite_difference():
    d = gen.config(0, walk_num=2)
    basis = O.Basis(d)
    pts = gen.points(d)
    nucl = np.array(d["nucl_coord"])
    coef = d["mo_coef"]
    rng = np.random.default_rng(7)
    w = rng.standard_normal((pts.shape[0], 5, coef.shape[0]))
    gc, gn, gr = O.mo_vgl_adjoint(basis, pts, nucl, coef, w)
    h = 1.0e-4
    fd = np.zeros_like(gn)
    for a in range(nucl.shape[1]):
        for k in range(3):
            tp, tm = nucl.copy(), nucl.copy()
            tp[k, a] += h
            tm[k, a] -= h
            fd[a, k] = (_loss(basis, coef, w, pts, tp) - _loss(basis, coef, w, pts, tm)) / (2 * h)
    assert np.abs(fd - gn).max() < 1e-6 * np.abs(gn).max()
    # translation invariance: moving every nucleus and every point together
    # leaves L unchanged
    assert np.abs(gn.sum(axis=0) + gr.sum(axis=0)).max() < 1e-9 * np.abs(gn).max()
    # L is linear in the coefficients
    av = O.ao_vgl(basis, pts, nucl, path="doc")
    ref = np.einsum("pci,pck->ik", w, av)
    assert np.abs(gc - ref).max() < 1e-12 * np.abs(ref).max()


def test_orbital_forces_match_nuclear_finite_differences(chbrclf, basis):
    """The reference's forces tests (org/qmckl_forces.org:5800-5917, 6370-6480, 6780-6880):
    forces_mo_value / _mo_g / _mo_l against a 9-point finite difference of mo_value /
    the MO gradient rows / the MO Laplacian rows over the nuclear coordinates
    (step 1e-5, |diff| < 1e-9); forces_ao_value is minus the AO gradient on each nucleus."""
    pts = chbrclf["elec_coord"][0][:12]
    nucl = np.array(chbrclf["nucl_coord"], dtype=np.float64)
    coef = chbrclf["mo_coef"]
    N, P, M = nucl.shape[1], pts.shape[0], coef.shape[0]
    fao, fmv, fmg, fml = O.forces(basis, pts, nucl, coef)
    dx = 1.0e-5
    fd_v = np.zeros((N, P, 3, M))
    fd_g = np.zeros((N, 3, P, 3, M))
    fd_l = np.zeros((N, 3, P, M))
    for a in range(N):
        for k in range(3):
            for m in range(-4, 5):
                if m == 0:
                    continue
                t = nucl.copy()
                t[k, a] += m * dx
                mo = O.mo_vgl(coef, O.ao_vgl(basis, pts, t, path="doc"))     # [P][5][M]
                w = STENCIL[m + 4] / dx
                fd_v[a, :, k, :] += w * mo[:, 0, :]
                fd_g[a, k] += w * mo[:, 1:4, :]
                fd_l[a, k] += w * mo[:, 4, :]
    assert np.abs(fd_v - fmv).max() < 1e-9
    assert np.abs(fd_g - fmg).max() < 1e-9
    assert np.abs(fd_l - fml).max() < 1e-9
    av = O.ao_vgl(basis, pts, nucl, path="doc")
    for a in range(N):
        s0, ns = int(chbrclf["nucleus_index"][a]), int(chbrclf["nucleus_shell_num"][a])
        mask = np.zeros(basis.ao_num, bool)
        k = 0
        for s in range(chbrclf["shell_ang_mom"].size):
            l = int(chbrclf["shell_ang_mom"][s])
            nk = (l + 1) * (l + 2) // 2
            if s0 <= s < s0 + ns:
                mask[k:k + nk] = True
            k += nk
        assert np.array_equal(fao[a][:, :, mask], -av[:, 1:4, mask])
        assert not fao[a][:, :, ~mask].any()
