"""Batched MO VGL: many independent systems in one persistent launch.

* every system's slice of the batched result agrees with the single-system
  mixed evaluation of its own context to the mixed-form bound (the
  single-system fused kernel contracts the AOs in its own K order, see
  fused_tc.cu, so the two differ by rounding);
* the per-system launch loop gives the same numbers;
* every (producer warps, queue order) variant of the autotuner gives the same
  numbers, the tuner's choice is written to and read back from the tuning
  file;
* the CUDA-graph replay sees new coordinates in the same buffers;
* a dependency wait capped at one poll, with the point-order items kept from
  publishing, ends the launch with an error status instead of hanging, and
  the batch works again afterwards;
* accuracy against the FP64 form (<= 1e-6 per component).
"""
import os

import numpy as np
import pytest

from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

from conftest import comp_error

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_case():
    import torch
    systems = gen.batch_config(num_systems=12, seed=20260102, max_walkers=24)
    systems.append(gen.config(0, walk_num=3))
    ctxs = [make_context(s, points=False, form=pq.FORM_MIXED) for s in systems]
    P = [gen.points(s).shape[0] for s in systems]
    P.append(0)                      # an empty system
    ctxs.append(make_context(systems[0], points=False, form=pq.FORM_MIXED))
    systems.append(systems[0])
    b = pq.b200_batch_create(ctxs, P)
    co, oo, (ct, ot) = pq.b200_batch_layout(b, len(ctxs))
    coord = np.zeros(ct)
    for s, sysd in enumerate(systems):
        if P[s]:
            coord[co[s]:co[s] + 3 * P[s]] = gen.points(sysd)[:P[s]].T.reshape(-1)
    d_coord = torch.tensor(coord, dtype=torch.float64, device="cuda")
    d_out = torch.zeros(ot, dtype=torch.float64, device="cuda")
    yield dict(systems=systems, ctxs=ctxs, P=P, b=b, co=co, oo=oo, coord=coord, d_coord=d_coord, d_out=d_out)
    pq.b200_batch_destroy(b)
    for c in ctxs:
        pq.context_destroy(c)


def _single(case, s, form=pq.FORM_MIXED):
    import torch
    sysd, P = case["systems"][s], case["P"][s]
    M = sysd["mo_num"]
    ctx = case["ctxs"][s] if form == pq.FORM_MIXED else make_context(sysd, points=False, form=form)
    c = case["coord"][case["co"][s]:case["co"][s] + 3 * P]
    dc = torch.tensor(c, dtype=torch.float64, device="cuda")
    out = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    pq.b200_synchronize(ctx)
    if form != pq.FORM_MIXED:
        pq.context_destroy(ctx)
    return out.cpu().numpy().reshape(P, 5, M)


def _slice(case, out, s):
    P, M = case["P"][s], case["systems"][s]["mo_num"]
    o = case["oo"][s]
    return out[o:o + 5 * P * M].reshape(P, 5, M)


def _run(case, loop=False):
    b = case["b"]
    case["d_out"].zero_()
    if loop:
        pq.b200_batch_mo_vgl_loop_device(b, case["d_coord"].data_ptr(), case["d_out"].data_ptr())
    else:
        pq.b200_batch_mo_vgl_device(b, case["d_coord"].data_ptr(), case["d_out"].data_ptr())
        assert pq.b200_batch_synchronize(b) == 0
    return case["d_out"].cpu().numpy()


def _check_equal_single(case, out):
    for s in range(len(case["systems"])):
        if case["P"][s] == 0:
            continue
        ref = _single(case, s)
        got = _slice(case, out, s)
        assert max(comp_error(got, ref)) <= 1e-6, s


def test_batch_matches_single_system(batch_case):
    out = _run(batch_case)
    _check_equal_single(batch_case, out)


def test_loop_matches_persistent(batch_case):
    a = _run(batch_case)
    b = _run(batch_case, loop=True)
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()


def test_every_tuning_variant(batch_case, tmp_path):
    b = batch_case["b"]
    ref = _run(batch_case)
    for pw in (16, 8):
        for order in (0, 1, 2):
            pq.b200_batch_set_tuning(b, pw, order)
            got = _run(batch_case)
            assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), (pw, order)
    tune = tmp_path / "tune.txt"
    os.environ["QMCKL_B200_TUNE_FILE"] = str(tune)
    try:
        best = pq.b200_batch_tune(b, batch_case["d_coord"].data_ptr(), batch_case["d_out"].data_ptr(), 2)
        assert best > 0
        choice = pq.b200_batch_get_tuning(b)
        assert tune.read_text().strip().startswith("batch ")
        b2 = pq.b200_batch_create(batch_case["ctxs"], batch_case["P"])
        assert pq.b200_batch_get_tuning(b2) == choice
        pq.b200_batch_destroy(b2)
    finally:
        del os.environ["QMCKL_B200_TUNE_FILE"]
    _check_equal_single(batch_case, _run(batch_case))


def test_graph_replay_sees_new_coordinates(batch_case):
    pq.b200_batch_set_graph(batch_case["b"], True)
    first = _run(batch_case)
    saved = batch_case["d_coord"].clone()
    batch_case["d_coord"].add_(0.05)
    batch_case["coord"] = batch_case["d_coord"].cpu().numpy()
    second = _run(batch_case)
    assert np.abs(second - first).max() > 0
    _check_equal_single(batch_case, second)
    batch_case["d_coord"].copy_(saved)
    batch_case["coord"] = saved.cpu().numpy()


def test_dependency_wait_cap_reports_failure(batch_case):
    b = batch_case["b"]
    pq.b200_batch_set_wait_limit(b, 1, publish=False)
    pq.b200_batch_mo_vgl_device(b, batch_case["d_coord"].data_ptr(), batch_case["d_out"].data_ptr())
    status = pq.b200_batch_synchronize(b, raise_on_error=False)
    assert status == 26
    with pytest.raises(RuntimeError):
        pq.b200_batch_synchronize(b)
    pq.b200_batch_set_wait_limit(b, 0, publish=True)
    _check_equal_single(batch_case, _run(batch_case))


def test_batch_accuracy_vs_fp64(batch_case):
    out = _run(batch_case)
    for s in (0, 5, len(batch_case["systems"]) - 2):
        if batch_case["P"][s] == 0:
            continue
        ref = _single(batch_case, s, form=pq.FORM_FP64)
        assert max(comp_error(_slice(batch_case, out, s), ref)) <= 1e-6
