"""The allocation-free MO VGL entry point against the regular ones (GPU).

Collected last on purpose (file name), so a failure here comes after every
other test has run.  It must pass both alone in a fresh process and after the
other tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import comp_error
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6


def _noalloc(ctx, npts, d_coord, d_out):
    f = pq.lib().qmckl_b200_mo_vgl_device_noalloc
    f.restype = C.c_int32
    return f(C.c_int64(ctx), C.c_int64(npts), C.c_void_p(d_coord), C.c_void_p(d_out))


def test_noalloc_matches_regular_entry_points_twice():
    """Two calls in a row: each within the mixed-form bound of the regular
    mixed evaluation and of the FP64 form, and neither changes the free
    device memory (the first call included)."""
    import torch
    d = gen.config(1, walk_num=1)                       # 318 points, 2000 AOs, 160 MOs
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    refs = {}
    for name, form in (("fp64", pq.FORM_FP64), ("mixed", pq.FORM_MIXED)):
        c = make_context(d, points=False, form=form)
        r = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
        pq.b200_mo_vgl_device(c, P, dc.data_ptr(), r.data_ptr())
        pq.b200_synchronize(c)
        refs[name] = r.cpu().numpy().reshape(P, 5, M)
        pq.context_destroy(c)
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    warm = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), warm.data_ptr())   # regular call: uploads, allocates
    pq.b200_synchronize(ctx)
    outs = [torch.full((P * 5 * M,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    free = []
    for o in outs:
        rc = _noalloc(ctx, P, dc.data_ptr(), o.data_ptr())
        assert rc == 0, pq.last_error(ctx)
        pq.b200_synchronize(ctx)
        free.append(torch.cuda.mem_get_info()[0])
    assert free == [free0, free0]
    for o in outs:
        h = o.cpu().numpy().reshape(P, 5, M)
        assert np.isfinite(h).all()
        assert max(comp_error(h, refs["mixed"])) < MIXED_TOL
        assert max(comp_error(h, refs["fp64"])) < MIXED_TOL
    pq.context_destroy(ctx)


def test_noalloc_rejects_oversize_and_unprepared():
    import torch
    d = gen.config(1, walk_num=2)                       # 636 points > 546-point limit
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    out = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    assert _noalloc(ctx, 4, dc.data_ptr(), out.data_ptr()) == 106          # not prepared yet
    pq.b200_mo_vgl_device(ctx, 4, dc.data_ptr(), out.data_ptr())          # prepare with a small call
    assert _noalloc(ctx, P, dc.data_ptr(), out.data_ptr()) == 2            # QMCKL_INVALID_ARG_2
    assert "at most 546 points" in pq.last_error(ctx)
    assert _noalloc(ctx, 1 << 62, dc.data_ptr(), out.data_ptr()) == 2      # no overflow in the size check
    assert _noalloc(ctx, 546, dc.data_ptr(), out.data_ptr()) == 0
    pq.b200_synchronize(ctx)
    pq.context_destroy(ctx)
