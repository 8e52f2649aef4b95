"""Parity of the CUDA path with the CPU oracle, through the C ABI (GPU)."""
import numpy as np
import pytest

from conftest import comp_error, parity_error
from oracle import pyoracle as O
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12   # parity_error bar of the FP64 form


@pytest.fixture(scope="module")
def chb(chbrclf):
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    yield chbrclf, ctx
    pq.context_destroy(ctx)


def test_golden_vectors_through_capi(chbrclf):
    """The reference's golden vectors, 68 points of walker 1 (org/qmckl_ao.org:4675-4712, 5223-5252, 9302-9384)."""
    d = dict(chbrclf)
    d["elec_coord"] = d["elec_coord"][:1]
    ctx = make_context(d, form=pq.FORM_FP64)
    P, Pn, S, A = 68, 297, 72, 263
    prim = pq.get_ao_basis_primitive_vgl(ctx, P * 5 * Pn).reshape(P, 5, Pn)
    shell = pq.get_ao_basis_shell_vgl(ctx, P * 5 * S).reshape(P, 5, S)
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    aval = pq.get_ao_basis_ao_value(ctx, P * A).reshape(P, A)
    for name, arr in (("prim_vgl", prim), ("shell_vgl", shell), ("ao_vgl", ao), ("ao_value", aval)):
        idx = d[f"golden_{name}_index"]
        got = np.array([arr[tuple(i)] for i in idx])
        assert np.all(np.abs(got - d[f"golden_{name}_value"]) < d[f"golden_{name}_tol"]), name
    pq.context_destroy(ctx)


def test_ao_vgl_chbrclf(chb):
    d, ctx = chb
    P, A = 136, 263
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    ref = O.ao_vgl(O.Basis(d), gen.points(d), d["nucl_coord"])
    assert parity_error(ao, ref) < FP64_TOL


def test_primitive_and_shell_vgl_chbrclf(chb):
    d, ctx = chb
    P = 136
    b = O.Basis(d)
    prim = pq.get_ao_basis_primitive_vgl(ctx, P * 5 * 297).reshape(P, 5, 297)
    ref = O.primitive_vgl(b, gen.points(d), d["nucl_coord"])
    assert np.abs(prim - ref).max() <= 1e-15 * max(1.0, np.abs(ref).max())
    shell = pq.get_ao_basis_shell_vgl(ctx, P * 5 * 72).reshape(P, 5, 72)
    ref = O.shell_vgl(b, gen.points(d), d["nucl_coord"])
    assert parity_error(shell, ref) < FP64_TOL


def test_mo_vgl_and_value_chbrclf(chb):
    d, ctx = chb
    P, A, M = 136, 263, 224
    b = O.Basis(d)
    ref_ao = O.ao_vgl(b, gen.points(d), d["nucl_coord"])
    ref = O.mo_vgl(d["mo_coef"], ref_ao)
    mo = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    assert parity_error(mo, ref) < FP64_TOL
    mv = pq.get_mo_basis_mo_value(ctx, P * M).reshape(P, M)
    assert np.abs(mv - mo[:, 0, :]).max() < 1e-12           # org/qmckl_mo.org:3745-3761
    pq.context_touch(ctx)
    mv2 = pq.get_mo_basis_mo_value(ctx, P * M).reshape(P, M)   # recomputed from AO values
    assert np.abs(mv2 - mo[:, 0, :]).max() < 1e-12
    ref_val = O.mo_value(d["mo_coef"], O.ao_value(b, gen.points(d), d["nucl_coord"]))
    assert parity_error(mv2, ref_val) < FP64_TOL


def test_inplace_and_rescale(chbrclf):
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    P, A, M = 136, 263, 224
    mo = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M)
    mo_in = pq.get_mo_basis_mo_vgl_inplace(ctx, P * 5 * M)
    assert np.array_equal(mo, mo_in)
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A)
    ao_in = pq.get_ao_basis_ao_vgl_inplace(ctx, P * 5 * A)
    assert np.array_equal(ao, ao_in)
    pq.mo_basis_rescale(ctx, 2.0)                             # org/qmckl_mo.org:3763-3781
    mv = pq.get_mo_basis_mo_value(ctx, P * M).reshape(P, M)
    assert np.abs(2.0 * mo.reshape(P, 5, M)[:, 0, :] - mv).max() < 1e-12
    pq.context_destroy(ctx)


def test_select_mo(chbrclf):
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    P, M = 136, 224
    full = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    keep = np.zeros(M, dtype=np.int32)
    keep[::3] = 1
    pq.mo_basis_select_mo(ctx, keep)
    m = int(keep.sum())
    sel = pq.get_mo_basis_mo_vgl(ctx, P * 5 * m).reshape(P, 5, m)
    assert np.array_equal(sel, full[:, :, keep.astype(bool)]) or parity_error(sel, full[:, :, keep.astype(bool)]) < 1e-14
    pq.context_destroy(ctx)


def test_moving_nuclei_needs_touch(chbrclf):
    """Nuclear coordinates do not touch the context; a touch recomputes (org/qmckl_mo.org:3937-3941)."""
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    P, A = 136, 263
    a0 = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A)
    nc = chbrclf["nucl_coord"].copy()
    nc[0, 0] += 0.1
    pq.set_nucleus_coord(ctx, "T", nc.reshape(-1))
    a1 = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A)
    assert np.array_equal(a0, a1)
    pq.context_touch(ctx)
    a2 = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    ref = O.ao_vgl(O.Basis(chbrclf), gen.points(chbrclf), nc)
    assert parity_error(a2, ref) < FP64_TOL
    pq.context_destroy(ctx)


def test_config0_parity():
    d = gen.config(0)
    ctx = make_context(d, form=pq.FORM_FP64)
    P, A, M = 1920, d["ao_num"], d["mo_num"]
    b = O.Basis(d)
    ref_ao = O.ao_vgl(b, gen.points(d), d["nucl_coord"])
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    assert parity_error(ao, ref_ao) < FP64_TOL
    mo = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    assert parity_error(mo, O.mo_vgl(d["mo_coef"], ref_ao)) < FP64_TOL
    pq.context_destroy(ctx)


def test_config1_subset_parity():
    """Config-1 molecule (2000 AOs, 160 MOs) on 8 walkers (2,544 points)."""
    d = gen.config(1, walk_num=8)
    ctx = make_context(d, form=pq.FORM_FP64)
    P, A, M = d["elec_coord"].shape[0] * d["elec_coord"].shape[1], d["ao_num"], d["mo_num"]
    b = O.Basis(d)
    ref_ao = O.ao_vgl(b, gen.points(d), d["nucl_coord"])
    mo = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    assert parity_error(ao, ref_ao) < FP64_TOL
    assert parity_error(mo, O.mo_vgl(d["mo_coef"], ref_ao)) < FP64_TOL
    pq.context_destroy(ctx)


@pytest.mark.parametrize("npts", [1, 7, 33])
def test_ragged_point_counts(chbrclf, npts):
    pts = gen.points(chbrclf)[:npts]
    ctx = make_context(chbrclf, points=False, form=pq.FORM_FP64)
    pq.set_point(ctx, "N", npts, pts.reshape(-1))
    A, M = 263, 224
    ao = pq.get_ao_basis_ao_vgl(ctx, npts * 5 * A).reshape(npts, 5, A)
    ref = O.ao_vgl(O.Basis(chbrclf), pts, chbrclf["nucl_coord"])
    assert parity_error(ao, ref) < FP64_TOL
    mo = pq.get_mo_basis_mo_vgl(ctx, npts * 5 * M).reshape(npts, 5, M)
    assert parity_error(mo, O.mo_vgl(chbrclf["mo_coef"], ref)) < FP64_TOL
    pq.context_destroy(ctx)


def test_single_precision_exponential_path(chbrclf):
    """precision 23: FP32 exponentials and the shorter cutoff, as the reference's SP branch."""
    ctx = make_context(chbrclf, form=pq.FORM_FP64, precision=23)
    P, A = 136, 263
    ao = pq.get_ao_basis_ao_vgl(ctx, P * 5 * A).reshape(P, 5, A)
    ref = O.ao_vgl(O.Basis(chbrclf), gen.points(chbrclf), chbrclf["nucl_coord"], precision=23)
    assert max(comp_error(ao, ref)) < 1e-6
    pq.context_destroy(ctx)


def test_device_entry_points(chbrclf):
    import torch
    ctx = make_context(chbrclf, points=False, form=pq.FORM_FP64)
    pts = gen.points(chbrclf)
    P, A, M = pts.shape[0], 263, 224
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    ao = torch.empty(P * 5 * A, dtype=torch.float64, device="cuda")
    mo = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    pq.b200_ao_vgl_device(ctx, P, dc.data_ptr(), ao.data_ptr())
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), mo.data_ptr())
    pq.b200_synchronize(ctx)
    ref_ao = O.ao_vgl(O.Basis(chbrclf), pts, chbrclf["nucl_coord"])
    assert parity_error(ao.cpu().numpy().reshape(P, 5, A), ref_ao) < FP64_TOL
    assert parity_error(mo.cpu().numpy().reshape(P, 5, M), O.mo_vgl(chbrclf["mo_coef"], ref_ao)) < FP64_TOL
    pq.context_destroy(ctx)


def test_kernels_were_launched(chbrclf):
    n0 = pq.b200_kernel_launch_count()
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    pq.get_mo_basis_mo_vgl(ctx, 136 * 5 * 224)
    assert pq.b200_kernel_launch_count() >= n0 + 2
    pq.context_destroy(ctx)
