"""MO counts at the edges of the tensor-core tiling (GPU).

The mixed form's kernels cut the MOs into N tiles of at most 160 columns,
rounded up to multiples of 16, and stage each output row for one bulk copy
only when the row length is even; the FP64 contraction uses 80-column tiles.
These counts cover one MO, counts just below and above a multiple of 16, an
odd count, and counts that take two and three N tiles, on the config-1
molecule (2000 AOs) for one walker (318 points), against the oracle.
"""
import numpy as np
import pytest

from conftest import comp_error, parity_error
from oracle import pyoracle as O
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-6


@pytest.fixture(scope="module")
def molecule():
    base = gen.config(1, walk_num=1)
    pts = gen.points(base)
    ao = O.ao_vgl(O.Basis(base), pts, base["nucl_coord"])
    return base, ao


def _with_mos(base, m, seed):
    d = dict(base)
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((base["ao_num"], m)))
    d["mo_coef"] = np.ascontiguousarray(q.T)
    d["mo_num"] = m
    return d


def _mo_vgl(d, form, fused=1):
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    ctx = make_context(d, form=form)
    if form == pq.FORM_MIXED:
        pq.b200_set_mixed_kernel(ctx, fused)
    try:
        return pq.get_mo_basis_mo_vgl(ctx, P * 5 * d["mo_num"]).reshape(P, 5, d["mo_num"])
    finally:
        pq.context_destroy(ctx)


@pytest.mark.parametrize("m", [1, 15, 17, 75, 161, 330])
def test_mo_counts(molecule, m):
    base, ao = molecule
    d = _with_mos(base, m, 7000 + m)
    ref = O.mo_vgl(d["mo_coef"], ao)
    assert parity_error(_mo_vgl(d, pq.FORM_FP64), ref) < FP64_TOL
    for fused in (1, 0):
        mo = _mo_vgl(d, pq.FORM_MIXED, fused)
        assert np.isfinite(mo).all()
        assert max(comp_error(mo, ref)) < MIXED_TOL, (m, fused)
