"""AO Hessian getter and MO VGL adjoint on the GPU, against the oracle and
against finite differences.

* qmckl_get_ao_basis_ao_hessian vs the oracle's restatement of
  qmckl_compute_ao_hessian_doc (FP64, parity metric <= 1e-12).
* qmckl_b200_mo_vgl_adjoint_device vs the oracle's orbital-forces
  contraction (FP64, <= 1e-10 of the largest entry).
* The adjoint-workload (config-1 molecule, 128 walkers, 40,704 points) with
  L = sum W * mo_vgl, W ~ N(0, 1): nuclear gradient against central finite
  differences of the FP64 forward (h = 1e-4 bohr); coefficient gradient
  against W^T AO; both FP64 and mixed forms; through torch.autograd too.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

from conftest import parity_error

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    return torch


def test_ao_hessian_getter_matches_oracle(chbrclf):
    ctx = make_context(chbrclf, form=pq.FORM_FP64)
    P = chbrclf["elec_coord"].shape[0] * chbrclf["elec_coord"].shape[1]
    A = chbrclf["ao_num"]
    got = pq.get_ao_basis_ao_hessian(ctx, 12 * P * A).reshape(3, P, 4, A)
    ref = O.ao_hessian(O.Basis(chbrclf), gen.points(chbrclf), chbrclf["nucl_coord"])
    pq.context_destroy(ctx)
    assert parity_error(got, ref) <= 1e-12


def test_ao_hessian_config0():
    d = gen.config(0, walk_num=8)
    ctx = make_context(d, form=pq.FORM_FP64)
    P, A = gen.points(d).shape[0], d["ao_num"]
    got = pq.get_ao_basis_ao_hessian(ctx, 12 * P * A).reshape(3, P, 4, A)
    ref = O.ao_hessian(O.Basis(d), gen.points(d), d["nucl_coord"])
    pq.context_destroy(ctx)
    assert parity_error(got, ref) <= 1e-12


def _adjoint(ctx, d, w, torch):
    pts = gen.points(d)
    P = pts.shape[0]
    M, A, N = d["mo_num"], d["ao_num"], d["nucl_num"]
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    dw = torch.tensor(w, dtype=torch.float64, device="cuda")
    gc = torch.empty((M, A), dtype=torch.float64, device="cuda")
    gn = torch.empty((N, 3), dtype=torch.float64, device="cuda")
    gr = torch.empty((3, P), dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_adjoint_device(ctx, P, dc.data_ptr(), dw.data_ptr(), gc.data_ptr(), gn.data_ptr(), gr.data_ptr())
    pq.b200_synchronize(ctx)
    return gc.cpu().numpy(), gn.cpu().numpy(), gr.cpu().numpy().T


def test_adjoint_matches_oracle_forces():
    torch = _torch()
    d = gen.config(0, walk_num=4)
    pts = gen.points(d)
    w = np.random.default_rng(11).standard_normal((pts.shape[0], 5, d["mo_num"]))
    ctx = make_context(d, points=False, form=pq.FORM_FP64)
    gc, gn, gr = _adjoint(ctx, d, w, torch)
    pq.context_destroy(ctx)
    rc, rn, rr = O.mo_vgl_adjoint(O.Basis(d), pts, d["nucl_coord"], d["mo_coef"], w)
    for got, ref in ((gc, rc), (gn, rn), (gr, rr)):
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_adjoint_partial_outputs_and_empty():
    torch = _torch()
    d = gen.config(0, walk_num=2)
    pts = gen.points(d)
    P = pts.shape[0]
    w = np.random.default_rng(3).standard_normal((P, 5, d["mo_num"]))
    ctx = make_context(d, points=False, form=pq.FORM_FP64)
    gc, gn, gr = _adjoint(ctx, d, w, torch)
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    dw = torch.tensor(w, dtype=torch.float64, device="cuda")
    only_n = torch.empty((d["nucl_num"], 3), dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_adjoint_device(ctx, P, dc.data_ptr(), dw.data_ptr(), 0, only_n.data_ptr(), 0)
    only_r = torch.empty((3, P), dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_adjoint_device(ctx, P, dc.data_ptr(), dw.data_ptr(), 0, 0, only_r.data_ptr())
    empty_n = torch.full((d["nucl_num"], 3), 7.0, dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_adjoint_device(ctx, 0, dc.data_ptr(), dw.data_ptr(), 0, empty_n.data_ptr(), 0)
    pq.b200_synchronize(ctx)
    pq.context_destroy(ctx)
    assert np.abs(only_n.cpu().numpy() - gn).max() <= 1e-12 * np.abs(gn).max()
    assert np.abs(only_r.cpu().numpy().T - gr).max() <= 1e-12 * np.abs(gr).max()
    assert float(empty_n.abs().max()) == 0.0


@pytest.fixture(scope="module")
def adjoint_case():
    """The adjoint workload: config-1 molecule, 128 walkers (40,704 points)."""
    d = gen.config(3)
    pts = gen.points(d)
    w = np.random.default_rng(20260003).standard_normal((pts.shape[0], 5, d["mo_num"]))
    return d, pts, w


def _fd_nuclear(d, pts, w, form, atoms, h=1.0e-4):
    """Central differences of L over the coordinates of `atoms` (FP64 forward on the GPU)."""
    torch = _torch()
    P, M = pts.shape[0], d["mo_num"]
    ctx = make_context(d, points=False, form=form)
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    dw = torch.tensor(w, dtype=torch.float64, device="cuda")
    out = torch.empty((P, 5, M), dtype=torch.float64, device="cuda")
    nucl = np.array(d["nucl_coord"], dtype=np.float64)   # [3][N]

    def loss(nc):
        pq.set_nucleus_coord(ctx, "T", nc.reshape(-1))
        pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
        pq.b200_synchronize(ctx)
        return float((dw * out).sum())

    fd = np.zeros((len(atoms), 3))
    for j, a in enumerate(atoms):
        for k in range(3):
            tp, tm = nucl.copy(), nucl.copy()
            tp[k, a] += h
            tm[k, a] -= h
            fd[j, k] = (loss(tp) - loss(tm)) / (2 * h)
    pq.context_destroy(ctx)
    return fd


def test_adjoint_matches_oracle_on_adjoint_molecule(adjoint_case):
    torch = _torch()
    d, pts, w = adjoint_case
    sub = dict(d)
    sub["elec_coord"] = pts[:400].reshape(1, -1, 3)
    ws = w[:400]
    ctx = make_context(sub, points=False, form=pq.FORM_FP64)
    gc, gn, gr = _adjoint(ctx, sub, ws, torch)
    pq.context_destroy(ctx)
    rc, rn, rr = O.mo_vgl_adjoint(O.Basis(d), pts[:400], d["nucl_coord"], d["mo_coef"], ws)
    for got, ref in ((gc, rc), (gn, rn), (gr, rr)):
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_adjoint_nuclear_gradient_fp64_vs_finite_differences(adjoint_case):
    torch = _torch()
    d, pts, w = adjoint_case
    ctx = make_context(d, points=False, form=pq.FORM_FP64)
    gc, gn, gr = _adjoint(ctx, d, w, torch)
    pq.context_destroy(ctx)
    atoms = list(range(d["nucl_num"]))
    fd = _fd_nuclear(d, pts, w, pq.FORM_FP64, atoms, h=1.0e-4)
    fd2 = _fd_nuclear(d, pts, w, pq.FORM_FP64, atoms, h=0.5e-4)
    scale = np.abs(gn).max()
    # the h = 1e-4 stencil itself errs by O(h^2) times the third derivative,
    # large near the tight (a ~ 5e3) primitives; Richardson's combination of
    # two steps removes the h^2 term
    err_h = np.abs(fd - gn).max() / scale
    err_r = np.abs((4.0 * fd2 - fd) / 3.0 - gn).max() / scale
    print(f"nuclear gradient: FD(h=1e-4) {err_h:.2e}, Richardson {err_r:.2e}")
    assert err_h <= 1e-4, err_h
    assert err_r <= 1e-6, err_r
    # translation invariance of L: sum of nuclear and point gradients vanishes
    assert np.abs(gn.sum(axis=0) + gr.sum(axis=0)).max() <= 1e-9 * np.abs(gn).max()


def test_adjoint_coefficient_gradient_fp64(adjoint_case):
    torch = _torch()
    d, pts, w = adjoint_case
    ctx = make_context(d, points=False, form=pq.FORM_FP64)
    gc, _, _ = _adjoint(ctx, d, w, torch)
    P, A = pts.shape[0], d["ao_num"]
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    ao = torch.empty((P, 5, A), dtype=torch.float64, device="cuda")
    pq.b200_ao_vgl_device(ctx, P, dc.data_ptr(), ao.data_ptr())
    pq.b200_synchronize(ctx)
    pq.context_destroy(ctx)
    ref = torch.einsum("pci,pck->ik", torch.tensor(w, device="cuda"), ao).cpu().numpy()
    assert np.abs(gc - ref).max() <= 1e-11 * np.abs(ref).max()


def test_adjoint_mixed_vs_fp64_finite_differences(adjoint_case):
    torch = _torch()
    d, pts, w = adjoint_case
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    gc, gn, gr = _adjoint(ctx, d, w, torch)
    pq.context_destroy(ctx)
    atoms = list(range(0, d["nucl_num"], 8))
    fd = _fd_nuclear(d, pts, w, pq.FORM_FP64, atoms, h=1.0e-4)
    fd2 = _fd_nuclear(d, pts, w, pq.FORM_FP64, atoms, h=0.5e-4)
    err = np.abs((4.0 * fd2 - fd) / 3.0 - gn[atoms]).max() / np.abs(gn).max()
    print(f"mixed nuclear gradient vs FP64 Richardson FD: {err:.2e}")
    assert err <= 1e-5, err
    ctx = make_context(d, points=False, form=pq.FORM_FP64)
    gc64, gn64, gr64 = _adjoint(ctx, d, w, torch)
    pq.context_destroy(ctx)
    # split-bfloat16 contractions (FP32 accumulation in K slices of 2048
    # rows, slices summed in FP64) and FP32 AO arithmetic: the same 1e-6 bar
    # as the forward mixed form
    for got, ref in ((gc, gc64), (gn, gn64), (gr, gr64)):
        assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("walkers,electrons", [(7, None), (1, 3)])
def test_adjoint_mixed_small_and_ragged(walkers, electrons):
    """Mixed adjoint on config-0 sizes (90 AOs, 90 MOs: one 128-column MO
    tile) with row counts that are not multiples of the 32-row stage, and on 3
    points (15 rows, fewer than one tile), against the oracle."""
    torch = _torch()
    d = gen.config(0, walk_num=walkers)
    if electrons is not None:
        d = dict(d)
        d["elec_coord"] = d["elec_coord"][:, :electrons]
    pts = gen.points(d)
    w = np.random.default_rng(11).standard_normal((pts.shape[0], 5, d["mo_num"]))
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    got = _adjoint(ctx, d, w, torch)
    pq.context_destroy(ctx)
    ref = O.mo_vgl_adjoint(O.Basis(d), pts, d["nucl_coord"], d["mo_coef"], w)
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() <= 1e-6 * np.abs(r).max()


def test_autograd_function(adjoint_case):
    torch = _torch()
    from qmckl_b200 import torch_ops
    d, pts, w = adjoint_case
    pts = pts[:4096]
    w = w[:4096]
    ctx = make_context(d, points=False, form=pq.FORM_FP64)
    coord = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda", requires_grad=True)
    nucl = torch_ops.nucl_coord_tensor(d).requires_grad_(True)
    coef = torch.tensor(d["mo_coef"], dtype=torch.float64, requires_grad=True)
    W = torch.tensor(w, dtype=torch.float64, device="cuda")
    mo = torch_ops.mo_vgl(ctx, coord, nucl, coef)
    loss = (W * mo).sum()
    loss.backward()
    # the same numbers through the C ABI directly
    sub = dict(d)
    sub["elec_coord"] = pts.reshape(1, -1, 3)
    gc, gn, gr = _adjoint(ctx, sub, w, torch)
    assert np.abs(coef.grad.numpy() - gc).max() <= 1e-12 * np.abs(gc).max()
    assert np.abs(nucl.grad.numpy() - gn).max() <= 1e-12 * np.abs(gn).max()
    assert np.abs(coord.grad.cpu().numpy().T - gr).max() <= 1e-12 * np.abs(gr).max()
    # a point-coordinate derivative by central differences through the Function
    h = 1e-4
    with torch.no_grad():
        for (i, k) in ((0, 0), (17, 1), (4095, 2)):
            cp = coord.detach().clone()
            cm = coord.detach().clone()
            cp[k, i] += h
            cm[k, i] -= h
            fd = (float((W * torch_ops.mo_vgl(ctx, cp, nucl, coef)).sum()) -
                  float((W * torch_ops.mo_vgl(ctx, cm, nucl, coef)).sum())) / (2 * h)
            g = float(coord.grad[k, i])
            assert abs(fd - g) <= 1e-5 * float(coord.grad.abs().max())
    torch_ops.forget(ctx)
    pq.context_destroy(ctx)


def test_adjoint_mixed_two_mo_tiles():
    """250 MOs: two MO tiles in both tensor-core contractions of the mixed
    adjoint (dL/dC: tiles of 192 MOs; G = W C^T: K = 250 in 4 K blocks),
    against the oracle on 60 points of the config-1 molecule."""
    torch = _torch()
    d = dict(gen.config(1, walk_num=1))
    rng = np.random.default_rng(17)
    q, _ = np.linalg.qr(rng.standard_normal((d["ao_num"], 250)))
    d["mo_coef"] = np.ascontiguousarray(q.T)
    d["mo_num"] = 250
    d["elec_coord"] = d["elec_coord"][:, :60]
    pts = gen.points(d)
    w = rng.standard_normal((pts.shape[0], 5, 250))
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    got = _adjoint(ctx, d, w, torch)
    pq.context_destroy(ctx)
    ref = O.mo_vgl_adjoint(O.Basis(d), pts, d["nucl_coord"], d["mo_coef"], w)
    for g, r in zip(got, ref):
        assert np.abs(g - r).max() <= 1e-6 * np.abs(r).max()
