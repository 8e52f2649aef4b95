"""The device entry points return before the GPU finishes, and a bounded
barrier wait that gives up is reported at the next synchronization point
(GPU).

No GPU fault is involved: the failure is written into the context's error
word by the test hook, the same word a timed-out wait of the tensor-core
kernels sets.
"""
import numpy as np
import pytest

from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

pytestmark = pytest.mark.gpu


def _setup(fused=1):
    import torch
    d = gen.config(1, walk_num=8)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    pq.b200_set_mixed_kernel(ctx, fused)
    stream = torch.cuda.Stream()
    pq.b200_set_stream(ctx, stream.cuda_stream)
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    return d, P, M, ctx, stream, dc


@pytest.mark.parametrize("fused", [1, 0])
def test_device_entry_returns_before_the_gpu_finishes(fused):
    import torch
    d, P, M, ctx, stream, dc = _setup(fused)
    ref = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), ref.data_ptr())     # first call: uploads the tables
    pq.b200_synchronize(ctx)
    outs = [torch.full((P * 5 * M,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        torch.cuda._sleep(400_000_000)          # ~0.2 s of a spinning kernel ahead of the evaluations
    for o in outs:
        pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), o.data_ptr())
    busy = not stream.query()                   # the host is back while the stream still works
    pq.b200_synchronize(ctx)
    assert busy
    for o in outs:
        assert torch.equal(o, ref)
    pq.context_destroy(ctx)


def test_wait_failure_is_reported_at_the_next_synchronization():
    import torch
    d, P, M, ctx, stream, dc = _setup()
    out = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    pq.b200_synchronize(ctx)
    good = out.clone()
    # enqueueing still succeeds; the synchronization reports the failure once
    pq.b200_inject_wait_failure(ctx, 13)
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    with pytest.raises(RuntimeError, match="bounded barrier wait"):
        pq.b200_synchronize(ctx)
    pq.b200_synchronize(ctx)                    # cleared: the context stays usable
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    pq.b200_synchronize(ctx)
    assert torch.equal(out, good)
    pq.context_destroy(ctx)


def test_wait_failure_is_reported_by_the_host_getter():
    d = gen.config(1, walk_num=2)
    P, M = d["elec_coord"].shape[0] * d["elec_coord"].shape[1], d["mo_num"]
    ctx = make_context(d, form=pq.FORM_MIXED)
    good = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M)
    pq.b200_inject_wait_failure(ctx, 11)
    with pytest.raises(RuntimeError, match="bounded barrier wait"):
        pq.get_mo_basis_mo_vgl(ctx, P * 5 * M)
    assert np.array_equal(pq.get_mo_basis_mo_vgl(ctx, P * 5 * M), good)
    pq.context_destroy(ctx)


@pytest.mark.parametrize("cfg", [0, 1])
def test_late_warps_leave_the_results_unchanged(cfg):
    """Producer warps holding a chunk of a skipped 16-AO k-step sleep before
    their stage wait (test hook), so the MMAs of their block, and on the
    two-block tiles of config 0 (three stages) every MMA of the tile, can
    complete before that wait starts: a parity wait alone would then wait for
    a stage use that never comes.  The fused kernel ends such waits on the
    count of released blocks: no wait gives up and the results are the same
    to the last bit."""
    import torch
    d = gen.config(0) if cfg == 0 else gen.config(1, walk_num=2)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    ctx = make_context(d, points=False, form=pq.FORM_MIXED)
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    out = torch.full((P * 5 * M,), float("nan"), dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    pq.b200_synchronize(ctx)
    good = out.clone()
    evaluated, total = pq.b200_get_kblock_stats(ctx, reset=True)
    assert 0 < evaluated < total   # some k-steps are skipped
    pq.b200_inject_late_warps(100_000)
    try:
        for _ in range(3):
            out.fill_(float("nan"))
            pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
            pq.b200_synchronize(ctx)   # raises if a bounded wait gave up
            assert torch.equal(out, good)
    finally:
        pq.b200_inject_late_warps(0)
    pq.context_destroy(ctx)
