"""The standalone AO helpers of the C API (host code, CPU only).

qmckl_ao_power, qmckl_ao_gaussian_vgl and the five cartesian-monomial
functions (org/qmckl_ao.org:3804-3910, 5937-6026, 6195-6914) against:

* the oracle's restatement of the monomial tables (oracle_poly_vgl, both
  the HPC form and the doc form), bit for bit, lmax 0..7;
* the reference's own compiled qmckl_ao_polynomial_transp_vgl_hpc
  (oracle/_ref, where the reference's sources were present at build time),
  bit for bit, lmax 0..12, several leading dimensions;
* the checks of the reference's own tests (test_qmckl_ao_power,
  test_qmckl_ao_gaussian_vgl, test_qmckl_ao_polynomial_vgl: the same inputs,
  the same relative tolerances);
* the reference's exit codes for each invalid argument.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as O
from oracle import refpath
from qmckl_b200 import qmckl as pq

# Fortran's default-real literals (1.1, 2.2, ...) in the reference's tests are
# single precision, widened to double.
X_TEST = np.array([1.1, 2.2, 3.3], dtype=np.float32).astype(np.float64)
R_TEST = np.array([0.1, 1.2, -2.3], dtype=np.float32).astype(np.float64)


@pytest.fixture(scope="module")
def ctx():
    c = pq.context_create()
    yield c
    pq.context_destroy(c)


def _rc(name, *args):
    f = getattr(pq.lib(), name)
    f.restype = C.c_int32
    return f(*args)


def _points(seed=3, k=6):
    rng = np.random.default_rng(seed)
    return [(rng.uniform(-3, 3, 3), rng.uniform(-3, 3, 3)) for _ in range(k)]


# ------------------------------------------------------------ monomials


@pytest.mark.parametrize("lmax", range(0, O.MAX_L + 1))
def test_polynomials_match_oracle_bit_for_bit(ctx, lmax):
    for X, R in _points(seed=lmax) + [(X_TEST, R_TEST)]:
        hpc, n = O.poly_vgl(lmax, X, R, path="hpc")
        doc, n_doc = O.poly_vgl(lmax, X, R, path="doc")
        assert n == n_doc == (lmax + 1) * (lmax + 2) * (lmax + 3) // 6
        # transposed forms: VGL[5][ldv]
        for f in (pq.ao_polynomial_transp_vgl, pq.ao_polynomial_transp_vgl_hpc):
            m, L, V = f(ctx, X, R, lmax, ldv=n + 3)
            assert m == n
            assert np.array_equal(V[:, :n], hpc)
            assert not V[:, n:].any()
            assert np.array_equal(L, O.monomial_powers(lmax)[:n])
        # The doc forms differ from each other only by the 1e-20 shift of
        # X - R, which rounds away for these displacements.
        for f in (pq.ao_polynomial_vgl, pq.ao_polynomial_vgl_doc):
            m, L, V = f(ctx, X, R, lmax, ldl=4, ldv=7)
            assert m == n
            assert np.array_equal(V[:n, :5].T, doc)
            assert not V[:, 5:].any() and not L[:, 3:].any()
            assert np.array_equal(L[:n, :3], O.monomial_powers(lmax)[:n])
        m, L, V = pq.ao_polynomial_transp_vgl_doc(ctx, X, R, lmax)
        assert m == n and np.array_equal(V, doc)


def test_doc_shift_is_applied_to_the_displacement(ctx):
    """At X == R the non-transposed doc form evaluates at Y = 1e-20 (so x^1 is
    1e-20), the transposed doc form at Y = 0, and the HPC form adds 1e-20
    after the products (org/qmckl_ao.org:6283, 6541, 6845-6874)."""
    X = np.array([0.5, -0.25, 2.0])
    _, _, vdoc = pq.ao_polynomial_vgl(ctx, X, X, 3)
    _, _, vtd = pq.ao_polynomial_transp_vgl_doc(ctx, X, X, 3)
    _, _, vhpc = pq.ao_polynomial_transp_vgl_hpc(ctx, X, X, 3)
    assert vdoc[1, 0] == 1e-20 and vdoc[4, 0] == 1e-20 * 1e-20
    assert vtd[0, 1] == 0.0 and vtd[0, 4] == 0.0
    assert vhpc[0, 1] == 1e-20 and vhpc[0, 4] == 1e-20 and vhpc[0, 19] == 1e-20
    assert vhpc[0, 0] == vdoc[0, 0] == vtd[0, 0] == 1.0


def test_polynomial_vgl_reference_test(ctx):
    """test_qmckl_ao_polynomial_vgl (org/qmckl_ao.org:6942-7040): lmax 4,
    ldl 3, ldv 100, values and derivatives against Y**L within epsilon."""
    lmax, eps = 4, pq.get_numprec_epsilon(ctx)
    Y = X_TEST - R_TEST
    n, L, V = pq.ao_polynomial_vgl(ctx, X_TEST, R_TEST, lmax, ldl=3, ldv=100)
    assert n == 35 and (L >= 0).all()
    for j in range(n):
        a = L[j]
        mono = lambda e: np.prod([Y[i] ** e[i] for i in range(3)])  # noqa: E731
        assert abs(1 - V[j, 0] / mono(a)) <= eps
        w = 0.0
        for i in range(3):
            if a[i] < 1:
                assert V[j, 1 + i] == 0.0
            else:
                e = a.copy()
                e[i] -= 1
                assert abs(1 - V[j, 1 + i] / (a[i] * mono(e))) <= eps
            if a[i] > 1:
                e = a.copy()
                e[i] -= 2
                w += a[i] * (a[i] - 1) * mono(e)
        if w != 0.0:
            assert abs(1 - V[j, 4] / w) <= eps


def _ref_hpc():
    L = refpath.lib()
    f = L.qmckl_ao_polynomial_transp_vgl_hpc
    f.restype = C.c_int32
    f.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                  C.c_int64]
    return f


@pytest.mark.skipif(not refpath.available(), reason="oracle/_ref not built (no reference sources)")
@pytest.mark.parametrize("lmax", range(0, 13))
def test_transp_hpc_matches_the_reference_bit_for_bit(ctx, lmax):
    ref = _ref_hpc()
    npoly = (lmax + 1) * (lmax + 2) * (lmax + 3) // 6
    # ldv == 4 and ldv == 50 take table-copy branches in the reference
    for ldl, ldv in ((3, npoly), (5, npoly + 1), (3, 4 if lmax == 1 else 50 if lmax == 2 else npoly + 7)):
        for X, R in _points(seed=100 + lmax, k=4):
            out = []
            for which in ("mine", "ref"):
                L = np.full((npoly, ldl), -7, dtype=np.int32)
                V = np.full((5, ldv), -3.0)
                n = C.c_int64(-1)
                args = (X.ctypes.data_as(C.c_void_p), R.ctypes.data_as(C.c_void_p), lmax, C.byref(n),
                        L.ctypes.data_as(C.c_void_p), ldl, V.ctypes.data_as(C.c_void_p), ldv)
                if which == "mine":
                    rc = _rc("qmckl_ao_polynomial_transp_vgl_hpc", C.c_int64(ctx), *args[:2], C.c_int32(lmax),
                             args[3], args[4], C.c_int64(ldl), args[6], C.c_int64(ldv))
                else:
                    rc = ref(1, *args)
                assert rc == 0
                out.append((n.value, L, V))
            (n0, L0, V0), (n1, L1, V1) = out
            assert n0 == n1 == npoly
            assert np.array_equal(L0[:, :3], L1[:, :3])
            if lmax == 2 and ldv == 50:
                # The reference's lmax-2 shortcut for ldv == 50 copies a packed
                # 5 x 10 table (stride 10, not ldv; org/qmckl_ao.org:6744-6758).
                # This library keeps the stride-ldv layout of every other case.
                assert np.array_equal(V1.ravel()[:50], V0[:, :10].ravel())
                continue
            assert np.array_equal(V0[:, :npoly], V1[:, :npoly]), (lmax, ldl, ldv)


@pytest.mark.skipif(not refpath.available(), reason="oracle/_ref not built (no reference sources)")
def test_transp_hpc_error_codes_match_the_reference(ctx):
    ref = _ref_hpc()
    X, R = X_TEST, R_TEST
    L = np.zeros((400, 8), dtype=np.int32)
    V = np.zeros(5 * 400)
    n = C.c_int64(0)
    for lmax, ldl, ldv in ((-1, 3, 10), (2, 2, 10), (0, 3, 0), (1, 3, 3), (2, 3, 9), (3, 3, 19), (5, 3, 55),
                           (5, 3, 56), (3, 3, 20)):
        args = (X.ctypes.data_as(C.c_void_p), R.ctypes.data_as(C.c_void_p))
        mine = _rc("qmckl_ao_polynomial_transp_vgl_hpc", C.c_int64(ctx), *args, C.c_int32(lmax), C.byref(n),
                   L.ctypes.data_as(C.c_void_p), C.c_int64(ldl), V.ctypes.data_as(C.c_void_p), C.c_int64(ldv))
        theirs = ref(1, *args, lmax, C.byref(n), L.ctypes.data_as(C.c_void_p), ldl, V.ctypes.data_as(C.c_void_p),
                     ldv)
        assert mine == theirs, (lmax, ldl, ldv)


def test_polynomial_error_codes(ctx):
    X, R = X_TEST.ctypes.data_as(C.c_void_p), R_TEST.ctypes.data_as(C.c_void_p)
    L = np.zeros((100, 4), dtype=np.int32)
    V = np.zeros(5 * 100)
    Lp, Vp = L.ctypes.data_as(C.c_void_p), V.ctypes.data_as(C.c_void_p)
    n = C.c_int64(0)

    def rc(name, c=ctx, x=X, lmax=2, np_=C.byref(n), lp=Lp, ldl=3, vp=Vp, ldv=10):
        return _rc(name, C.c_int64(c), x, R, C.c_int32(lmax), np_, lp, C.c_int64(ldl), vp, C.c_int64(ldv))

    for name in ("qmckl_ao_polynomial_vgl", "qmckl_ao_polynomial_vgl_doc", "qmckl_ao_polynomial_transp_vgl",
                 "qmckl_ao_polynomial_transp_vgl_doc", "qmckl_ao_polynomial_transp_vgl_hpc"):
        assert rc(name) == 0 and n.value == 10
        assert rc(name, c=0) == 103                 # QMCKL_INVALID_CONTEXT
        assert rc(name, lmax=-1) == 4
        assert rc(name, lmax=1001) == 4
        assert rc(name, ldl=2) == 7
        assert rc(name, ldv=4) == 9                 # < 5 (doc) and < 10 monomials (transposed)
        assert rc(name, x=None) == 2
        assert rc(name, np_=None) == 5
        assert rc(name, lp=None) == 6
        assert rc(name, vp=None) == 8
    # the non-transposed form needs ldv >= 5 only; the transposed forms need
    # ldv >= the number of monomials
    assert rc("qmckl_ao_polynomial_vgl", lmax=4, ldv=5) == 0
    assert rc("qmckl_ao_polynomial_transp_vgl_doc", lmax=4, ldv=34) == 9
    assert rc("qmckl_ao_polynomial_transp_vgl_doc", lmax=4, ldv=35) == 0


def test_high_lmax_beyond_the_oracle(ctx):
    """lmax up to 20: the monomial count, the order and the values against
    Y**L (relative 1e-13), all three forms."""
    X, R = np.array([0.7, -1.3, 0.4]), np.array([-0.2, 0.1, 1.1])
    Y = X - R
    for lmax in (8, 12, 20):
        npoly = (lmax + 1) * (lmax + 2) * (lmax + 3) // 6
        for f in (pq.ao_polynomial_transp_vgl_hpc, pq.ao_polynomial_transp_vgl_doc):
            n, L, V = f(ctx, X, R, lmax)
            assert n == npoly
            deg = L.sum(axis=1)
            assert (np.diff(deg) >= 0).all()
            expect = np.prod(Y[None, :] ** L, axis=1)
            assert np.allclose(V[0], expect, rtol=1e-13, atol=1e-19)
        n, L, V = pq.ao_polynomial_vgl(ctx, X, R, lmax)
        assert n == npoly and np.allclose(V[:, 0], np.prod(Y[None, :] ** L[:, :3], axis=1), rtol=1e-13)


# ---------------------------------------------------------------- powers


def test_ao_power_reference_test(ctx):
    """test_qmckl_ao_power (org/qmckl_ao.org:6054-6094): n 100, ldp 10."""
    n, ldp = 100, 10
    j = np.arange(1, n + 1)
    X = -5.0 + 0.1 * j
    LMAX = (1 + j % 5).astype(np.int32)
    P = pq.ao_power(ctx, X, LMAX, ldp)
    eps = 3 * pq.get_numprec_epsilon(ctx)
    for i in range(n):
        for k in range(1, LMAX[i] + 1):
            e = X[i] ** k
            assert (P[i, k - 1] == 0.0) if e == 0.0 else abs(1 - P[i, k - 1] / e) <= eps
        assert not P[i, LMAX[i]:].any()
        # running products, bit for bit
        assert np.array_equal(P[i, :LMAX[i]], np.cumprod(np.full(LMAX[i], X[i])))


def test_ao_power_error_codes(ctx):
    X = np.linspace(-1, 1, 12)
    P = np.zeros((12, 8))

    def rc(c=ctx, n=12, lmax=(3,) * 12, ldp=8):
        lm = np.array(lmax, dtype=np.int32)
        return _rc("qmckl_ao_power", C.c_int64(c), C.c_int64(n), X.ctypes.data_as(C.c_void_p),
                   lm.ctypes.data_as(C.c_void_p), P.ctypes.data_as(C.c_void_p), C.c_int64(ldp))

    assert rc() == 0
    assert rc(c=0) == 103
    assert rc(ldp=12) == 2 and rc(ldp=20) == 2      # n <= ldp, as in the reference
    assert rc(lmax=(9,) + (3,) * 11) == 6           # ldp < max(LMAX)
    assert rc(lmax=(0,) * 12) == 4                  # max(LMAX) <= 0
    assert rc(lmax=(0,) * 11 + (1,)) == 0
    assert rc(n=0, ldp=-1) == 4


# ------------------------------------------------------------- Gaussians


def test_gaussian_vgl_reference_test(ctx):
    """test_qmckl_ao_gaussian_vgl (org/qmckl_ao.org:3931-4008): n 10, ldv 100,
    A_i = 0.0013 * 2^i, relative error <= 3 epsilon."""
    n, ldv = 10, 100
    A = float(np.float32(0.0013)) * np.array([2.0 ** i for i in range(1, n + 1)])
    V = pq.ao_gaussian_vgl(ctx, X_TEST, R_TEST, A, ldv=ldv)
    Y = X_TEST - R_TEST
    r2 = (Y ** 2).sum()
    eps = 3 * pq.get_numprec_epsilon(ctx)
    g = np.exp(-A * r2)
    assert np.all(np.abs(1 - V[0, :n] / g) <= eps)
    for d in range(3):
        assert np.all(np.abs(1 - V[1 + d, :n] / (-2 * A * Y[d] * g)) <= eps)
    assert np.all(np.abs(1 - V[4, :n] / (A * (4 * r2 * A - 6) * g)) <= eps)
    assert not V[:, n:].any()


def test_gaussian_vgl_error_codes(ctx):
    A = np.ones(4)
    V = np.zeros(5 * 8)
    Xp, Rp = X_TEST.ctypes.data_as(C.c_void_p), R_TEST.ctypes.data_as(C.c_void_p)

    def rc(c=ctx, n=4, ldv=8, a=A.ctypes.data_as(C.c_void_p), v=V.ctypes.data_as(C.c_void_p)):
        return _rc("qmckl_ao_gaussian_vgl", C.c_int64(c), Xp, Rp, C.c_int64(n), a, v, C.c_int64(ldv))

    assert rc() == 0
    assert rc(c=0) == 103
    assert rc(n=0) == 4
    assert rc(ldv=3) == 7
    assert rc(a=None) == 5
    assert rc(v=None) == 6
