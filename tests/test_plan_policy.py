"""The fused kernel's MO tiling (host logic, CPU only).

qmckl_b200_get_fused_plan returns the tiling that mo_tc.cu's tc_plan_fused
chooses: with 3 pieces, MO tiles of up to 256 columns with two accumulators
when they take fewer tiles than tiles of up to 160, or as many tiles with
three A stages (tiles of up to 176 MOs, which fit 225 KB of shared memory);
three accumulators and two stages otherwise, for 2 pieces and under
QMCKL_B200_WIDE_TILES=0; wide tiles wherever they fit under =1.  bench.py
mirrors the tile width to count the MMA flops the kernel issues, so the two
must agree.
"""
import importlib.util
import os

import pytest

from conftest import ROOT
from qmckl_b200 import qmckl as pq


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# mo_num -> (n_tile, n_tiles, accumulators, stages), 3 pieces, default policy
DEFAULT = {
    16: (16, 1, 2, 3),
    90: (96, 1, 2, 3),
    160: (160, 1, 2, 3),    # config 1: one wide tile, three stages
    161: (176, 1, 2, 3),
    176: (176, 1, 2, 3),
    177: (192, 1, 2, 2),    # fewer tiles than two of 160, two stages only
    224: (224, 1, 2, 2),
    256: (256, 1, 2, 2),
    300: (160, 2, 2, 3),
    350: (176, 2, 2, 3),    # config 4
    400: (208, 2, 2, 2),
    500: (256, 2, 2, 2),
}


@pytest.fixture(autouse=True)
def _no_env(monkeypatch):
    monkeypatch.delenv("QMCKL_B200_WIDE_TILES", raising=False)


@pytest.mark.parametrize("mo", sorted(DEFAULT))
def test_default_tiling(mo):
    assert pq.b200_get_fused_plan(2000, mo, 3) == DEFAULT[mo]


@pytest.mark.parametrize("mo", sorted(DEFAULT))
def test_bench_mirrors_the_tile_width(mo):
    assert _bench().fused_n_tile(mo) == DEFAULT[mo][0]


@pytest.mark.parametrize("mo", [90, 160, 161, 224, 350, 500])
def test_narrow_tiling_with_two_pieces_and_when_forced(mo, monkeypatch):
    narrow_tiles = -(-mo // 160)
    narrow = (-(-(-(-mo // narrow_tiles)) // 16) * 16, narrow_tiles, 3, 2)
    assert pq.b200_get_fused_plan(2000, mo, 2) == narrow
    monkeypatch.setenv("QMCKL_B200_WIDE_TILES", "0")
    assert pq.b200_get_fused_plan(2000, mo, 3) == narrow


def test_wide_tiles_whenever_they_fit_when_forced(monkeypatch):
    monkeypatch.setenv("QMCKL_B200_WIDE_TILES", "1")
    assert pq.b200_get_fused_plan(2000, 160, 3) == (160, 1, 2, 3)
    assert pq.b200_get_fused_plan(2000, 224, 3) == (224, 1, 2, 2)


def test_invalid_arguments():
    for args, code in (((0, 160, 3), 1), ((2000, 0, 3), 2), ((2000, 160, 4), 3)):
        with pytest.raises(RuntimeError, match=f"Invalid argument {code}$"):
            pq.b200_get_fused_plan(*args)
