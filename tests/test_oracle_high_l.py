"""The oracle at angular momenta up to l = 7 (CPU only).

The reference evaluates cartesian polynomials of any degree and tests its two
polynomial kernels (doc and HPC) against each other for lmax = 0..7
(org/qmckl_ao.org:7042-7076) and against the closed form x^a y^b z^c for
lmax = 4 (6940-7040).  The same checks pin the oracle's restatements, and a
finite-difference check of the AO gradients and Laplacians pins the product
rule on a molecule with g, h, i and k shells.
"""
import numpy as np
import pytest

from conftest import parity_error
from oracle import pyoracle as O
from qmckl_b200 import gen


def test_polynomial_closed_form_lmax4():
    """Closed-form check of qmckl_ao_polynomial_vgl at lmax = 4
    (org/qmckl_ao.org:6940-7040): X = (1.1, 2.2, 3.3) and R = (0.1, 1.2, -2.3)
    as the Fortran test writes them (single-precision literals), relative
    error at most epsilon = 2^-52 for every monomial and component."""
    X = np.array([1.1, 2.2, 3.3], dtype=np.float32).astype(np.float64)
    R = np.array([0.1, 1.2, -2.3], dtype=np.float32).astype(np.float64)
    Y = X - R
    eps = 2.0 ** -52
    for path in ("doc", "hpc"):
        vgl, n = O.poly_vgl(4, X, R, path=path)
        assert n == 35
        for j, (a, b, c) in enumerate(O.monomial_powers(4)):
            L = (a, b, c)
            val = Y[0] ** a * Y[1] ** b * Y[2] ** c
            assert abs(1.0 - vgl[0, j] / val) <= eps, (path, L)
            for d in range(3):
                if L[d] < 1:
                    assert vgl[1 + d, j] == 0.0
                else:
                    e = list(L)
                    e[d] -= 1
                    g = L[d] * Y[0] ** e[0] * Y[1] ** e[1] * Y[2] ** e[2]
                    assert abs(1.0 - vgl[1 + d, j] / g) <= eps, (path, L, d)
            w = 0.0
            for d in range(3):
                if L[d] > 1:
                    e = list(L)
                    e[d] -= 2
                    w += L[d] * (L[d] - 1) * Y[0] ** e[0] * Y[1] ** e[1] * Y[2] ** e[2]
            if w != 0.0:
                assert abs(1.0 - vgl[4, j] / w) <= eps, (path, L)


@pytest.mark.parametrize("lmax", range(0, 8))
def test_polynomial_doc_and_hpc_agree(lmax):
    """doc and HPC polynomials for lmax = 0..7 at X = (1.1, 2.2, 3.3),
    R = (0.2, 1.1, 3.0): relative difference < 1e-15 with the reference's
    1e-100 guard (org/qmckl_ao.org:7042-7076)."""
    X = np.array([1.1, 2.2, 3.3])
    R = np.array([0.2, 1.1, 3.0])
    v0, n0 = O.poly_vgl(lmax, X, R, path="doc")
    v1, n1 = O.poly_vgl(lmax, X, R, path="hpc")
    assert n0 == n1 == (lmax + 1) * (lmax + 2) * (lmax + 3) // 6
    assert np.all(np.abs(1.0 - (v0 + 1e-100) / (v1 + 1e-100)) < 1e-15)


def test_oracle_rejects_l_above_7():
    d = gen.high_l_config(walk_num=1)
    d = dict(d)
    d["shell_ang_mom"] = d["shell_ang_mom"].copy()
    d["shell_ang_mom"][-1] = 8
    with pytest.raises(ValueError):
        O.Basis(d)


@pytest.fixture(scope="module")
def high_l():
    return gen.high_l_config(walk_num=4)


def test_high_l_hpc_and_doc_paths_agree(high_l):
    """AO VGL and MO VGL of the g/h/i/k molecule by the two restated algorithms."""
    b = O.Basis(high_l)
    pts = gen.points(high_l)
    h = O.ao_vgl(b, pts, high_l["nucl_coord"], path="hpc")
    d = O.ao_vgl(b, pts, high_l["nucl_coord"], path="doc")
    assert np.isfinite(h).all()
    assert parity_error(h, d) < 1e-13
    assert parity_error(O.mo_vgl(high_l["mo_coef"], h), O.mo_vgl(high_l["mo_coef"], d)) < 1e-12


def test_high_l_derivatives_by_finite_differences(high_l):
    """Gradient and Laplacian of every AO (l up to 7) against 4th-order
    central differences of the AO values (h = 1e-3 bohr), relative to each
    (point, component) row's largest entry."""
    b = O.Basis(high_l)
    pts = gen.points(high_l)[:24]
    N = high_l["nucl_coord"]
    h = 1e-3
    ao = O.ao_vgl(b, pts, N)
    grad = np.zeros((pts.shape[0], 3, b.ao_num))
    lap = np.zeros((pts.shape[0], b.ao_num))
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        v = {k: O.ao_vgl(b, pts + k * e, N)[:, 0, :] for k in (-2, -1, 1, 2)}
        grad[:, d, :] = (v[-2] - 8 * v[-1] + 8 * v[1] - v[2]) / (12 * h)
        lap += (-v[-2] + 16 * v[-1] - 30 * ao[:, 0, :] + 16 * v[1] - v[2]) / (12 * h * h)
    for d in range(3):
        s = np.abs(ao[:, 1 + d, :]).max(axis=1, keepdims=True)
        assert (np.abs(grad[:, d, :] - ao[:, 1 + d, :]) / s).max() < 1e-7
    s = np.abs(ao[:, 4, :]).max(axis=1, keepdims=True)
    assert (np.abs(lap - ao[:, 4, :]) / s).max() < 1e-5
