"""Cusp-adjusted MOs, MO Hessian and point-nucleus distances on the GPU,
against the oracle (whose restatement is pinned by the fit's defining
conditions and the reference's finite-difference tests, test_oracle_cusp.py).

* qmckl_set_mo_basis_r_cusp fits the cubics with this library's own getters
  (as the reference does with its own) and restores the caller's points;
  mo_vgl / mo_value then leave out the s AOs of a nucleus inside its radius
  and add its cubic: FP64 form <= 1e-12 (parity metric) against the oracle,
  mixed form <= 1e-6 per component (fused and unfused kernels, the device
  entry point and the no-allocation entry point);
* qmckl_get_mo_basis_mo_hessian, plain (CHBrClF) and cusp-adjusted, FP64;
* qmckl_get_electron_en_distance;
* select_mo fits the kept MOs again; batches and the adjoint refuse a
  context with r_cusp set.
"""
import ctypes

import numpy as np
import pytest

from oracle import pyoracle as O
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

from conftest import comp_error, parity_error
from test_oracle_cusp import cusp_system, near_nuclei

pytestmark = pytest.mark.gpu


def _ctx_with_points(d, pts, form):
    ctx = make_context(d, points=False, form=form)
    pq.set_point(ctx, "T", pts.shape[0], np.ascontiguousarray(pts.T).reshape(-1))
    return ctx


@pytest.fixture(scope="module")
def case():
    d, rc = cusp_system()
    pts = near_nuclei(d, rc, per=12)
    basis = O.Basis(d)
    prm = O.cusp_param(basis, d, rc)
    an, al = O.ao_nucl_ang_mom(d)
    nuc = np.asarray(d["nucl_coord"])
    ref_vgl = O.mo_vgl_cusp(d["mo_coef"], O.ao_vgl(basis, pts, nuc, path="doc"), an, al, pts, nuc, rc, prm)
    ref_val = O.mo_value_cusp(d["mo_coef"], O.ao_value(basis, pts, nuc), an, al, O.en_distance(pts, nuc), rc, prm)
    ref_hes = O.mo_hessian(d["mo_coef"], O.ao_hessian(basis, pts, nuc), an, al, pts, nuc, rc, prm)
    return dict(d=d, rc=rc, pts=pts, basis=basis, prm=prm, an=an, al=al, vgl=ref_vgl, val=ref_val, hes=ref_hes)


def test_set_r_cusp_restores_points(case):
    d, pts = case["d"], case["pts"]
    ctx = _ctx_with_points(d, pts, pq.FORM_FP64)
    pq.set_mo_basis_r_cusp(ctx, case["rc"])
    back = pq.get_point(ctx, "T", 3 * pts.shape[0]).reshape(3, -1).T
    assert np.array_equal(back, pts)
    pq.context_destroy(ctx)


def test_fp64_cusp_mo_vgl_value_hessian(case):
    d, pts = case["d"], case["pts"]
    P, M = pts.shape[0], d["mo_num"]
    ctx = _ctx_with_points(d, pts, pq.FORM_FP64)
    plain = pq.get_mo_basis_mo_vgl(ctx, 5 * P * M).reshape(P, 5, M)
    pq.set_mo_basis_r_cusp(ctx, case["rc"])
    vgl = pq.get_mo_basis_mo_vgl(ctx, 5 * P * M).reshape(P, 5, M)
    assert np.abs(vgl - plain).max() > 1e-3                  # the adjustment changes the MOs near the nuclei
    assert parity_error(vgl, case["vgl"]) <= 1e-12
    val = pq.get_mo_basis_mo_value(ctx, P * M).reshape(P, M)  # taken from the current mo_vgl
    assert parity_error(val, case["vgl"][:, 0, :]) <= 1e-12
    ctx2 = _ctx_with_points(d, pts, pq.FORM_FP64)
    pq.set_mo_basis_r_cusp(ctx2, case["rc"])
    val2 = pq.get_mo_basis_mo_value(ctx2, P * M).reshape(P, M)  # its own path
    assert parity_error(val2, case["val"]) <= 1e-12
    hes = pq.get_mo_basis_mo_hessian(ctx2, 9 * P * M).reshape(3, P, 3, M)
    assert parity_error(hes, case["hes"]) <= 1e-12
    # the AO getters still return the plain AOs
    av = pq.get_ao_basis_ao_vgl(ctx, 5 * P * d["ao_num"]).reshape(P, 5, -1)
    assert parity_error(av, O.ao_vgl(case["basis"], pts, d["nucl_coord"])) <= 1e-12
    pq.context_destroy(ctx)
    pq.context_destroy(ctx2)


@pytest.mark.parametrize("fused", [1, 0])
def test_mixed_cusp_mo_vgl(case, fused):
    d, pts = case["d"], case["pts"]
    P, M = pts.shape[0], d["mo_num"]
    ctx = _ctx_with_points(d, pts, pq.FORM_MIXED)
    pq.b200_set_mixed_kernel(ctx, fused)
    pq.set_mo_basis_r_cusp(ctx, case["rc"])
    vgl = pq.get_mo_basis_mo_vgl(ctx, 5 * P * M).reshape(P, 5, M)
    assert max(comp_error(vgl, case["vgl"])) <= 1e-6
    ctx2 = _ctx_with_points(d, pts, pq.FORM_MIXED)
    pq.b200_set_mixed_kernel(ctx2, fused)
    pq.set_mo_basis_r_cusp(ctx2, case["rc"])
    val = pq.get_mo_basis_mo_value(ctx2, P * M).reshape(P, M)
    assert max(comp_error(val[:, None, :], case["val"][:, None, :])) <= 1e-6
    pq.context_destroy(ctx)
    pq.context_destroy(ctx2)


def test_device_entries_with_cusp(case):
    import torch
    d, pts = case["d"], case["pts"]
    P, M = pts.shape[0], d["mo_num"]
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    for form, tol in ((pq.FORM_FP64, None), (pq.FORM_MIXED, 1e-6)):
        ctx = make_context(d, points=False, form=form)
        pq.set_mo_basis_r_cusp(ctx, case["rc"])
        out = torch.empty((P, 5, M), dtype=torch.float64, device="cuda")
        pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
        pq.b200_synchronize(ctx)
        got = out.cpu().numpy()
        if tol is None:
            assert parity_error(got, case["vgl"]) <= 1e-12
        else:
            assert max(comp_error(got, case["vgl"])) <= tol
            out2 = torch.zeros_like(out)
            f = pq.lib().qmckl_b200_mo_vgl_device_noalloc
            f.restype = ctypes.c_int32
            rc = f(ctypes.c_int64(ctx), ctypes.c_int64(P), ctypes.c_void_p(dc.data_ptr()),
                   ctypes.c_void_p(out2.data_ptr()))
            assert rc == 0
            assert max(comp_error(out2.cpu().numpy(), case["vgl"])) <= tol
        pq.context_destroy(ctx)


def test_plain_mo_hessian_chbrclf(chbrclf):
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    P = chbrclf["elec_coord"].shape[0] * chbrclf["elec_coord"].shape[1]
    M = chbrclf["mo_coef"].shape[0]
    got = pq.get_mo_basis_mo_hessian(ctx, 9 * P * M).reshape(3, P, 3, M)
    basis = O.Basis(chbrclf)
    ref = O.mo_hessian(chbrclf["mo_coef"], O.ao_hessian(basis, gen.points(chbrclf), chbrclf["nucl_coord"]))
    pq.context_destroy(ctx)
    assert parity_error(got, ref) <= 1e-12


def test_en_distance(case):
    d, pts = case["d"], case["pts"]
    ctx = _ctx_with_points(d, pts, pq.FORM_FP64)
    N = d["nucl_num"]
    got = pq.get_electron_en_distance(ctx, pts.shape[0] * N).reshape(-1, N)
    pq.context_destroy(ctx)
    assert np.abs(got - O.en_distance(pts, d["nucl_coord"])).max() <= 1e-15 * np.abs(got).max()


def test_select_mo_refits(case):
    d, pts = case["d"], case["pts"]
    P = pts.shape[0]
    keep = np.zeros(d["mo_num"], dtype=np.int32)
    keep[[0, 3, 7, 20]] = 1
    ctx = _ctx_with_points(d, pts, pq.FORM_FP64)
    pq.set_mo_basis_r_cusp(ctx, case["rc"])
    pq.mo_basis_select_mo(ctx, keep)
    got = pq.get_mo_basis_mo_vgl(ctx, 5 * P * 4).reshape(P, 5, 4)
    pq.context_destroy(ctx)
    sub = dict(d)
    sub["mo_coef"] = d["mo_coef"][keep == 1]
    prm = O.cusp_param(case["basis"], sub, case["rc"])
    nuc = np.asarray(d["nucl_coord"])
    ref = O.mo_vgl_cusp(sub["mo_coef"], O.ao_vgl(case["basis"], pts, nuc, path="doc"), case["an"], case["al"], pts,
                        nuc, case["rc"], prm)
    assert parity_error(got, ref) <= 1e-12


def test_batch_and_adjoint_refuse_cusp(case):
    import torch
    d = case["d"]
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    pq.set_mo_basis_r_cusp(ctx, case["rc"])
    with pytest.raises(RuntimeError):
        pq.b200_batch_create([ctx], [4])
    P, M, A, N = 4, d["mo_num"], d["ao_num"], d["nucl_num"]
    dc = torch.zeros((3, P), dtype=torch.float64, device="cuda")
    w = torch.zeros((P, 5, M), dtype=torch.float64, device="cuda")
    gn = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(RuntimeError):
        pq.b200_mo_vgl_adjoint_device(ctx, P, dc.data_ptr(), w.data_ptr(), 0, gn.data_ptr(), 0)
    pq.context_destroy(ctx)


def test_singular_radius_rejected(case):
    d = case["d"]
    ctx = make_context(d, points=False, form=pq.FORM_FP64)
    rc = np.array(case["rc"])
    rc[0] = 0.5            # 2 R Z - 6 = 0 for the carbon at index 0
    with pytest.raises(RuntimeError):
        pq.set_mo_basis_r_cusp(ctx, rc)
    pq.context_destroy(ctx)
