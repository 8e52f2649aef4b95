"""Inputs at the edges of what the library accepts, and the accuracy of the
mixed form under relative measures, against the CPU oracle (GPU).

* Angular momenta up to l = 7 (g, h, i, k shells): the FP64 form within the
  parity bar, the mixed form (fused and unfused kernels) within its bound.
* The config-4 shape (5000 AOs, 350 MOs: three MO tiles of the fused kernel)
  on a subset of its walkers.
* The mixed form's error measured three ways per component (value, three
  gradient components, Laplacian): max|diff| / max|ref|, the row-floored
  relative error of the FP64 parity metric, and the element-wise relative
  error over |ref| > 1e-8 max|ref|; plus the reference's own acceptance test
  for reduced precision, the average number of bits the result shares with
  the FP64 one (org/qmckl_mo.org:3798-3861).
"""
import numpy as np
import pytest

from conftest import (bits_of_agreement, comp_error, elementwise_rel_error, mixed_error_report, parity_error,
                      row_floored_error)
from oracle import pyoracle as O
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-6          # max |mixed - fp64| / max |fp64| per component
# Relative measures the mixed form meets (measured: row-floored <= 4.2e-4,
# element-wise <= 9e-2 over |ref| > 1e-8 max|ref|, 20.7-23.2 average bits;
# FP32 AO values and FP32 accumulation bound it, not the 1e-6 target)
MIXED_ROW_TOL = 1e-3
MIXED_ELEM_TOL = 0.2
MIXED_MIN_BITS = 20.0


def _oracle_mo(d, pts=None):
    pts = gen.points(d) if pts is None else pts
    ao = O.ao_vgl(O.Basis(d), pts, d["nucl_coord"])
    return O.mo_vgl(d["mo_coef"], ao), ao


def _eval(d, form, fused=1, pieces=3):
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    ctx = make_context(d, form=form)
    if form == pq.FORM_MIXED:
        pq.b200_set_mixed_kernel(ctx, fused)
        pq.b200_set_split_terms(ctx, pieces)
    try:
        return pq.get_mo_basis_mo_vgl(ctx, P * 5 * d["mo_num"]).reshape(P, 5, d["mo_num"])
    finally:
        pq.context_destroy(ctx)


@pytest.fixture(scope="module")
def high_l():
    d = gen.high_l_config(walk_num=16)
    ref_mo, ref_ao = _oracle_mo(d)
    return d, ref_mo, ref_ao


def test_high_l_fp64(high_l):
    """FP64 AO VGL, AO value, MO VGL and MO value with g, h, i, k shells."""
    d, ref_mo, ref_ao = high_l
    P, A, M = ref_ao.shape[0], d["ao_num"], d["mo_num"]
    ctx = make_context(d, form=pq.FORM_FP64)
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    assert parity_error(ao, ref_ao) < FP64_TOL
    av = pq.get_ao_basis_ao_value(ctx, P * A).reshape(P, A)
    assert parity_error(av, O.ao_value(O.Basis(d), gen.points(d), d["nucl_coord"])) < FP64_TOL
    mo = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    assert parity_error(mo, ref_mo) < FP64_TOL
    mv = pq.get_mo_basis_mo_value(ctx, P * M).reshape(P, M)
    assert parity_error(mv, ref_mo[:, 0, :]) < FP64_TOL
    pq.context_destroy(ctx)


def test_high_l_ao_hessian(high_l):
    d, _, _ = high_l
    pts = gen.points(d)[:64]
    dd = dict(d)
    dd["elec_coord"] = pts.reshape(1, -1, 3)
    dd["elec_up_num"], dd["elec_dn_num"] = 32, 32
    ctx = make_context(dd, form=pq.FORM_FP64)
    P, A = 64, d["ao_num"]
    h = pq.get_ao_basis_ao_hessian(ctx, 3 * P * 4 * A).reshape(3, P, 4, A)
    ref = O.ao_hessian(O.Basis(d), pts, d["nucl_coord"]).reshape(3, P, 4, A)
    assert parity_error(h, ref) < FP64_TOL
    pq.context_destroy(ctx)


@pytest.mark.parametrize("fused", [1, 0])
def test_high_l_mixed(high_l, fused):
    d, ref_mo, _ = high_l
    mo = _eval(d, pq.FORM_MIXED, fused=fused)
    assert np.isfinite(mo).all()
    assert max(comp_error(mo, ref_mo)) < MIXED_TOL, mixed_error_report(mo, ref_mo)


@pytest.fixture(scope="module")
def config4():
    d = gen.config(4, walk_num=4)          # 2,800 points, 5000 AOs, 350 MOs
    ref_mo, _ = _oracle_mo(d)
    return d, ref_mo


def test_config4_fp64(config4):
    d, ref_mo = config4
    mo = _eval(d, pq.FORM_FP64)
    assert parity_error(mo, ref_mo) < FP64_TOL


def test_config4_mixed_fused_three_mo_tiles(config4):
    """350 MOs: the fused kernel runs three MO tiles per point tile."""
    d, ref_mo = config4
    mo = _eval(d, pq.FORM_MIXED, fused=1)
    assert max(comp_error(mo, ref_mo)) < MIXED_TOL, mixed_error_report(mo, ref_mo)


@pytest.fixture(scope="module")
def mixed_cases(chbrclf):
    cases = {}
    for name, d in (("chbrclf", chbrclf), ("config0", gen.config(0)), ("config1_sub", gen.config(1, walk_num=16))):
        ref, _ = _oracle_mo(d)
        cases[name] = (ref, _eval(d, pq.FORM_MIXED))
    return cases


@pytest.mark.parametrize("name", ["chbrclf", "config0", "config1_sub"])
def test_mixed_error_measures(mixed_cases, name):
    """All three measures against the oracle (printed for the record with
    pytest -s): the max-normalised one within 1e-6, the row-floored and the
    element-wise relative errors within the bounds the form meets."""
    ref, mo = mixed_cases[name]
    rep = mixed_error_report(mo, ref)
    print(name, rep)
    assert max(comp_error(mo, ref)) < MIXED_TOL
    assert max(row_floored_error(mo, ref)) < MIXED_ROW_TOL
    assert max(elementwise_rel_error(mo, ref)) < MIXED_ELEM_TOL


@pytest.mark.parametrize("name", ["chbrclf", "config0", "config1_sub"])
def test_mixed_bits_of_agreement(mixed_cases, name):
    """The reference's single-precision acceptance test (org/qmckl_mo.org:3798-3861):
    the average number of bits the reduced-precision MO VGL shares with the
    FP64 one exceeds 11; this form keeps at least 20."""
    ref, mo = mixed_cases[name]
    bits = bits_of_agreement(mo, ref)
    print(name, "average bits", bits.mean(), "per component", bits.mean(axis=(0, 2)))
    assert bits.mean() > 11
    assert bits.mean(axis=(0, 2)).min() >= MIXED_MIN_BITS


def test_fp64_tile_sparse_contraction_ragged_and_far(chbrclf):
    """The FP64 form's tile-sparse contraction (spatial tiles of 25 points,
    each summing only the AOs of the shells that reach one of its points, in
    the basis order): point counts that end mid-tile,
    MO VGL and MO value through the device entry points, and points far from
    every nucleus (every block skipped: exact zeros)."""
    import torch
    ctx = make_context(chbrclf, points=False, form=pq.FORM_FP64)
    A, M = chbrclf["ao_num"], chbrclf["mo_num"]
    b = O.Basis(chbrclf)
    for npts in (1, 25, 26, 131):
        pts = gen.points(chbrclf)[:npts].copy()
        if npts == 26:
            pts[-1] += 300.0
        dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
        mo = torch.full((npts * 5 * M,), float("nan"), dtype=torch.float64, device="cuda")
        mv = torch.full((npts * M,), float("nan"), dtype=torch.float64, device="cuda")
        pq.b200_mo_vgl_device(ctx, npts, dc.data_ptr(), mo.data_ptr())
        pq.b200_mo_value_device(ctx, npts, dc.data_ptr(), mv.data_ptr())
        pq.b200_synchronize(ctx)
        ref = O.mo_vgl(chbrclf["mo_coef"], O.ao_vgl(b, pts, chbrclf["nucl_coord"]))
        got = mo.cpu().numpy().reshape(npts, 5, M)
        assert parity_error(got, ref) < FP64_TOL, npts
        refv = O.mo_value(chbrclf["mo_coef"], O.ao_value(b, pts, chbrclf["nucl_coord"]))
        assert parity_error(mv.cpu().numpy().reshape(npts, M), refv) < FP64_TOL, npts
        if npts == 26:
            assert not got[-1].any()
    pq.context_destroy(ctx)
