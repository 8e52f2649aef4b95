"""Mixed form (FP32 AOs, split 16-bit tcgen05 MO contraction) against the FP64 oracle (GPU).

Operand splits: 3 bfloat16 pieces (the default) or 2 float16 pieces of
power-of-two scaled values (22 significant bits instead of 24: on CHBrClF,
whose value rows cancel by up to 12x, that shows at ~1.2e-6).
"""
import numpy as np
import pytest

from conftest import comp_error
from oracle import pyoracle as O
from qmckl_b200 import gen
from qmckl_b200 import qmckl as pq
from qmckl_b200.system import make_context

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6       # max |mixed - fp64| / max |fp64| per component
MIXED_F16_CHBRCLF_TOL = 2e-6


def _mo_ref(d):
    ao = O.ao_vgl(O.Basis(d), gen.points(d), d["nucl_coord"])
    return O.mo_vgl(d["mo_coef"], ao), ao


@pytest.mark.parametrize("pieces,tol", [(3, MIXED_TOL), (2, MIXED_F16_CHBRCLF_TOL)])
def test_mixed_mo_vgl_chbrclf(chbrclf, pieces, tol):
    ctx = make_context(chbrclf, form=pq.FORM_MIXED)
    pq.b200_set_split_terms(ctx, pieces)
    P, M = 136, 224
    mo = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    ref, _ = _mo_ref(chbrclf)
    err = comp_error(mo, ref)
    assert max(err) < tol, err
    pq.context_destroy(ctx)


@pytest.mark.parametrize("fused", [0, 1])
def test_mixed_mo_value_chbrclf(chbrclf, fused):
    ctx = make_context(chbrclf, form=pq.FORM_MIXED)
    pq.b200_set_mixed_kernel(ctx, fused)
    P, M = 136, 224
    mv = pq.get_mo_basis_mo_value(ctx, P * M).reshape(P, M)
    ref, _ = _mo_ref(chbrclf)
    assert np.abs(mv - ref[:, 0, :]).max() / np.abs(ref[:, 0, :]).max() < MIXED_TOL
    pq.context_destroy(ctx)


@pytest.mark.parametrize("cid,walkers", [(0, 64), (1, 4)])
def test_mixed_configs(cid, walkers):
    d = gen.config(cid, walk_num=walkers)
    ctx = make_context(d, form=pq.FORM_MIXED)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    mo = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    ref, _ = _mo_ref(d)
    err = comp_error(mo, ref)
    assert max(err) < MIXED_TOL, err
    pq.context_destroy(ctx)


@pytest.mark.parametrize("fused,pieces", [(0, 2), (1, 2), (0, 3), (1, 3)])
def test_mixed_matches_fp64_gpu_on_config1_walkers(fused, pieces):
    """Mixed (both kernel organisations, both splits) vs the FP64 GPU form on 32 walkers of the config-1 molecule."""
    d = gen.config(1, walk_num=32)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    c64 = make_context(d, form=pq.FORM_FP64)
    c32 = make_context(d, form=pq.FORM_MIXED)
    pq.b200_set_mixed_kernel(c32, fused)
    pq.b200_set_split_terms(c32, pieces)
    a = pq.get_mo_basis_mo_vgl(c64, P * 5 * M).reshape(P, 5, M)
    b = pq.get_mo_basis_mo_vgl(c32, P * 5 * M).reshape(P, 5, M)
    assert max(comp_error(b, a)) < MIXED_TOL
    pq.context_destroy(c64)
    pq.context_destroy(c32)


def test_mixed_device_entry_and_ragged_rows(chbrclf):
    """Point counts whose 5*P rows end mid-tile (128-row tiles) and N tiles of the 224 MOs."""
    import torch
    ctx = make_context(chbrclf, points=False, form=pq.FORM_MIXED)
    for npts in (1, 25, 26, 131):
        pts = gen.points(chbrclf)[:npts]
        dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
        mo = torch.full((npts * 5 * 224,), float("nan"), dtype=torch.float64, device="cuda")
        pq.b200_mo_vgl_device(ctx, npts, dc.data_ptr(), mo.data_ptr())
        pq.b200_synchronize(ctx)
        got = mo.cpu().numpy().reshape(npts, 5, 224)
        ao = O.ao_vgl(O.Basis(chbrclf), pts, chbrclf["nucl_coord"])
        ref = O.mo_vgl(chbrclf["mo_coef"], ao)
        assert np.isfinite(got).all()
        # a handful of CHBrClF points: the value rows cancel by up to 12x
        # (sum_k |C A| / max |MO|), so the FP32 rounding shows at ~2e-6 here
        assert max(comp_error(got, ref)) < 5e-6
    pq.context_destroy(ctx)


def test_auto_form_follows_precision(chbrclf):
    """AUTO: FP64 at precision 53, mixed at precision <= 26."""
    P, M = 136, 224
    c1 = make_context(chbrclf)
    m1 = pq.get_mo_basis_mo_vgl(c1, P * 5 * M).reshape(P, 5, M)
    c2 = make_context(chbrclf, precision=26)
    m2 = pq.get_mo_basis_mo_vgl(c2, P * 5 * M).reshape(P, 5, M)
    ref, _ = _mo_ref(chbrclf)
    assert max(comp_error(m1, ref)) < 1e-13
    assert 1e-13 < max(comp_error(m2, ref)) < 1e-4
    pq.context_destroy(c1)
    pq.context_destroy(c2)


def test_host_getter_slices_match_device_entry():
    """The host getter evaluates large point sets in slices whose copies overlap the next slice's
    kernel; its result equals the device entry point's, to the last bit."""
    import torch
    d = gen.config(1, walk_num=64)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    M = d["mo_num"]
    ctx = make_context(d, form=pq.FORM_MIXED)
    host = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M)
    dc = torch.tensor(np.ascontiguousarray(gen.points(d).T), dtype=torch.float64, device="cuda")
    out = torch.empty(P * 5 * M, dtype=torch.float64, device="cuda")
    pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
    pq.b200_synchronize(ctx)
    assert np.array_equal(host, out.cpu().numpy())
    again = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M)   # cached: copied from the device array
    assert np.array_equal(host, again)
    pq.context_destroy(ctx)


def test_fused_tile_skipping():
    """The fused kernel orders its K dimension by shell radius class and
    nuclear position and skips the 64-AO blocks that vanish at every point of
    a tile.  Points far from every nucleus (all blocks skipped) give exact
    zeros; near points stay within the mixed-form bound of the FP64 form; the
    unfused kernels (basis order, no skipping) agree to the same bound."""
    import torch
    d = gen.config(1, walk_num=4)
    pts = gen.points(d)
    far = pts[:60] + 500.0
    allp = np.concatenate([pts, far])
    P, M = allp.shape[0], d["mo_num"]
    dc = torch.tensor(np.ascontiguousarray(allp.T), dtype=torch.float64, device="cuda")
    res = {}
    for name, form, fused in (("fp64", pq.FORM_FP64, 1), ("fused", pq.FORM_MIXED, 1), ("unfused", pq.FORM_MIXED, 0)):
        ctx = make_context(d, points=False, form=form)
        pq.b200_set_mixed_kernel(ctx, fused)
        out = torch.full((P, 5, M), 7.0, dtype=torch.float64, device="cuda")
        pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
        pq.b200_synchronize(ctx)
        res[name] = out.cpu().numpy()
        if name == "fused":
            ev, tot = pq.b200_get_kblock_stats(ctx, reset=True)
            # one count per CTA: ceil(P / 25) tiles x 1 MO tile, 32 K blocks of 4
            # k-steps each; the far points' tiles issue one (zero) block
            assert tot == -(-P // 25) * 32 * 4
            assert 0 < ev < tot
            assert pq.b200_get_kblock_stats(ctx) == (0, 0)
        pq.context_destroy(ctx)
    near = slice(0, pts.shape[0])
    assert not res["fused"][pts.shape[0]:].any()
    assert not res["fp64"][pts.shape[0]:].any()
    assert max(comp_error(res["fused"][near], res["fp64"][near])) <= MIXED_TOL
    assert max(comp_error(res["unfused"][near], res["fp64"][near])) <= MIXED_TOL


def test_fused_follows_precision_changes():
    """The fused kernel's K order and tile-skipping radii depend on the
    screening cutoff (ln 2^(p-1)): after the precision changes the mixed form
    agrees with the oracle at the new precision."""
    d = gen.config(0, walk_num=4)
    pts = gen.points(d)
    P, M = pts.shape[0], d["mo_num"]
    basis = O.Basis(d)
    ctx = make_context(d, form=pq.FORM_MIXED)
    first = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    ref53 = O.mo_vgl(d["mo_coef"], O.ao_vgl(basis, pts, d["nucl_coord"], precision=53))
    assert max(comp_error(first, ref53)) <= MIXED_TOL
    pq.set_numprec_precision(ctx, 30)
    second = pq.get_mo_basis_mo_vgl(ctx, P * 5 * M).reshape(P, 5, M)
    ref30 = O.mo_vgl(d["mo_coef"], O.ao_vgl(basis, pts, d["nucl_coord"], precision=30))
    assert max(comp_error(second, ref30)) <= MIXED_TOL
    pq.context_destroy(ctx)


@pytest.mark.parametrize("mos", [161, 330, 350])
def test_wide_mo_tiles(mos, monkeypatch):
    """Past 160 MOs the fused kernel takes MO tiles of up to 256 columns with
    two accumulators (leading product, corrections) and a single coefficient
    tile, so each AO is evaluated once per tile of 256 MOs rather than of
    160: one tile for 161 MOs, two for 330 and 350.  The results stay within
    the mixed-form bound of the FP64 form and of the three-accumulator tiling
    (QMCKL_B200_WIDE_TILES=0), and the kernel's statistics count the tiles it
    ran."""
    import torch
    d = gen.config(1, walk_num=2)
    rng = np.random.default_rng(10000 + mos)
    q, _ = np.linalg.qr(rng.standard_normal((d["ao_num"], mos)))
    d = dict(d, mo_coef=np.ascontiguousarray(q.T), mo_num=mos)
    pts = gen.points(d)
    P = pts.shape[0]
    dc = torch.tensor(np.ascontiguousarray(pts.T), dtype=torch.float64, device="cuda")
    res, tiles = {}, {}
    for name, form, wide in (("fp64", pq.FORM_FP64, "1"), ("wide", pq.FORM_MIXED, "1"), ("narrow", pq.FORM_MIXED, "0")):
        monkeypatch.setenv("QMCKL_B200_WIDE_TILES", wide)
        ctx = make_context(d, points=False, form=form)
        out = torch.full((P * 5 * mos,), float("nan"), dtype=torch.float64, device="cuda")
        pq.b200_mo_vgl_device(ctx, P, dc.data_ptr(), out.data_ptr())
        pq.b200_synchronize(ctx)
        res[name] = out.cpu().numpy().reshape(P, 5, mos)
        if form == pq.FORM_MIXED:
            _, tot = pq.b200_get_kblock_stats(ctx, reset=True)
            tiles[name] = tot // (-(-P // 25) * 32 * 4)
        pq.context_destroy(ctx)
    assert tiles["wide"] == -(-mos // 256)
    assert tiles["narrow"] == -(-mos // 160)
    assert np.isfinite(res["wide"]).all()
    assert max(comp_error(res["wide"], res["fp64"])) < MIXED_TOL
    assert max(comp_error(res["wide"], res["narrow"])) < MIXED_TOL


@pytest.mark.parametrize("mos", [224, 350])
def test_wide_mo_tiles_value_form(mos):
    """MO values alone (128-point tiles) with wide MO tiles: one tile of 224
    (two A stages) or two of 176 (three A stages where they fit, else the
    three-accumulator tiling), against the FP64 form, and the same values as
    the VGL form's value component within the mixed bound."""
    d = gen.config(1, walk_num=2)
    rng = np.random.default_rng(11000 + mos)
    q, _ = np.linalg.qr(rng.standard_normal((d["ao_num"], mos)))
    d = dict(d, mo_coef=np.ascontiguousarray(q.T), mo_num=mos)
    P = d["elec_coord"].shape[0] * d["elec_coord"].shape[1]
    res = {}
    for name, form in (("fp64", pq.FORM_FP64), ("mixed", pq.FORM_MIXED)):
        ctx = make_context(d, form=form)
        res[name] = pq.get_mo_basis_mo_value(ctx, P * mos).reshape(P, mos)
        if name == "mixed":
            res["vgl"] = pq.get_mo_basis_mo_vgl(ctx, P * 5 * mos).reshape(P, 5, mos)[:, 0, :]
        pq.context_destroy(ctx)
    scale = np.abs(res["fp64"]).max()
    assert np.isfinite(res["mixed"]).all()
    assert np.abs(res["mixed"] - res["fp64"]).max() / scale < MIXED_TOL
    assert np.abs(res["mixed"] - res["vgl"]).max() / scale < MIXED_TOL
