"""The allocation-free MO VGL entry point against the regular one (GPU).

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


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    d = gen.config(1, walk_num=1)                       # 318 points, 2000 AOs, 160 MOs
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    ref = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), ref.data_ptr())   # regular call: uploads, allocates
    pq.b200_synchronize(ctx)
    ref_h = ref.cpu().numpy().reshape(P, 5, M)
    outs = []
    free = []
    for _ in range(2):
        out = torch.full((P * 5 * M,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        rc = _noalloc(ctx, P, dc.data_ptr(), out.data_ptr())
        assert rc == 0, pq.last_error(ctx)
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy().reshape(P, 5, M))
    for o in outs:
        assert np.isfinite(o).all()
        assert max(comp_error(o, ref_h)) < MIXED_TOL
    # the second call allocates nothing on the device
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free[1]
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
    assert _noalloc(ctx, 546, dc.data_ptr(), out.data_ptr()) == 0
    pq.context_destroy(ctx)
