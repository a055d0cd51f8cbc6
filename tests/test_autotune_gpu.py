"""Tile-shape autotuner of the per-FO Coulomb kernel (flosic_sic_autotune),
through the C ABI.  The per-FO kernel's tiles are 128 mesh points by 32, 64 or
128 FO slots; the autotuner times each on the system's own Coulomb evaluation
and keeps the fastest.  The widths regroup FOs into CTAs without changing any
operation or its order, so a cycle after tuning must equal the untuned cycle
bit for bit, in FP64 and in the mixed mode, and each forced width must give
the same cycle as the default."""
import os

import numpy as np
import pytest

from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sysm():
    # 80 FOs: every width (32, 64, 128 slots) is a candidate
    return W.synthetic(natoms=10, nbasis=128, nmsh=20_000, nfo=80, box_ang=7.56, seed=1)


def same(a, b):
    assert a["esic"] == b["esic"]
    for key in ("results", "sic"):
        for s in range(len(a[key])):
            assert np.array_equal(a[key][s], b[key][s]), key
    assert np.array_equal(a["debdax"], b["debdax"])


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_autotune_keeps_results_bitwise(sysm, mode):
    ctx = S.open_system(sysm)
    try:
        ctx.set_precision(mode)
        ref = ctx.cycle()
        before = ctx.stats()
        width, times = ctx.autotune(reps=2)
        after = ctx.stats()
        assert width in (32, 64, 128)
        assert sorted(times) == [32, 64, 128]
        assert all(t > 0 for t in times.values())
        assert times[width] == min(times.values())
        # tuning runs leave the work counters and launch count alone
        for k in ("launches", "near_evals", "far_evals", "far_terms"):
            assert after[k] == before[k], k
        same(ctx.cycle(), ref)
    finally:
        ctx.close()


def test_forced_widths_agree(sysm, monkeypatch):
    cycles = []
    for wm in ("1", "2", "4"):
        monkeypatch.setenv("FLOSIC_PERFO_WM", wm)
        ctx = S.open_system(sysm)
        try:
            cycles.append(ctx.cycle())
        finally:
            ctx.close()
    same(cycles[0], cycles[1])
    same(cycles[0], cycles[2])


def test_autotune_skips_wide_tiles_for_few_fos():
    ctx = S.open_system(W.water(seed=0, nrad=12))
    try:
        width, times = ctx.autotune(reps=1)
        assert width == 32 and sorted(times) == [32]
    finally:
        ctx.close()


def test_autotune_argument_checks():
    ctx = S.open_system(W.water(seed=0, nrad=12))
    try:
        with pytest.raises(S.FlosicError):
            ctx.autotune(reps=0)
    finally:
        ctx.close()
    assert os.environ.get("FLOSIC_PERFO_WM") is None
