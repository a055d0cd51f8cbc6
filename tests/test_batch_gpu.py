"""C4 shape at test size: a batch of uneven alkane chains and rings
(workloads.alkane_batch), one context per molecule
(publicrelease_2020_b200.batch).  The batched cycle evaluates the Coulomb
potentials of all molecules in two persistent launches
(flosic_sic_batch_cycle); each molecule's result equals its own serial cycle
bit for bit, at every FO block width and in both precisions, and the
smallest molecules match the FP64 oracle at the parity tolerances of
tests/test_parity_gpu.py (LDA)."""
import time

import numpy as np
import pytest

from oracle import oracle as O
from publicrelease_2020_b200 import workloads as W
from publicrelease_2020_b200.batch import Batch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch():
    systems = W.alkane_batch(n=8, seed=100, max_carbons=5, nrad=(6, 10))
    b = Batch(systems)
    yield systems, b
    b.close()


def _same(systems, a, b, what):
    for s, p, q in zip(systems, a, b):
        assert p["esic"] == q["esic"], (what, s.name)
        for k in ("results", "sic", "debdax", "cfrm"):
            n = q[k].shape[1]
            assert np.array_equal(p[k][:, :n, ...][..., : q[k].shape[-1]], q[k]), (what, s.name, k)


def test_batched_launch_equals_serial_cycles(batch):
    systems, b = batch
    b.cycle()                       # first cycle: buffers allocated
    t0 = time.perf_counter()
    bat = b.cycle()
    t1 = time.perf_counter()
    ser = b.cycle_serial()
    t2 = time.perf_counter()
    con = b.cycle_streams()
    t3 = time.perf_counter()
    print(f"batch of {len(systems)}: batched launch {t1 - t0:.3f} s, serial {t2 - t1:.3f} s, "
          f"concurrent streams {t3 - t2:.3f} s")
    _same(systems, bat, ser, "batched")
    _same(systems, con, ser, "streams")


def test_batch_widths_and_autotune(batch):
    systems, b = batch
    ref = b.cycle_serial()
    for wm in (1, 2, 4):
        b.wm = wm
        _same(systems, b.cycle(), ref, f"wm={wm}")
    width, times = b.autotune(reps=1)
    assert width in (32, 64, 128) and set(times) == {32, 64, 128}
    _same(systems, b.cycle(), ref, "tuned")


def test_mixed_batch_equals_serial_mixed_cycles(monkeypatch):
    """Mixed precision: the batched launch runs the shared-geometry calls on
    the FP32-column FP64 GEMM, which the per-molecule path selects with
    FLOSIC_SHARED=mma; the two agree bit for bit."""
    monkeypatch.setenv("FLOSIC_SHARED", "mma")
    systems = W.alkane_batch(n=4, seed=120, max_carbons=4, nrad=(6, 8))
    b = Batch(systems, precision="mixed")
    try:
        _same(systems, b.cycle(), b.cycle_serial(), "mixed")
    finally:
        b.close()


def test_batch_molecules_match_oracle(batch):
    systems, b = batch
    res = b.cycle()
    order = sorted(range(len(systems)), key=lambda i: systems[i].nmsh * systems[i].nfrm[0])[:2]
    for i in order:
        s, g = systems[i], res[i]
        r = O.Oracle(s).sic_cycle(nthreads=8)
        assert abs(g["esic"] - r["esic"]) < 1e-9, s.name
        for sp in range(2):
            n = s.nfrm[sp]
            assert np.max(np.abs(g["results"][sp][:n, 1:] - r["results"][sp][:n, 1:])) < 1e-8, s.name
            lam_o = r["sic"][sp][:n, :n]
            assert np.max(np.abs(g["sic"][sp][:n, :n] - lam_o)) < 1e-9 * np.abs(lam_o).max(), s.name
            assert np.max(np.abs(g["debdax"][sp][:n] - r["debdax"][sp][:n])) < 1e-8 * max(
                1.0, np.abs(r["debdax"][sp][:n]).max()), s.name
