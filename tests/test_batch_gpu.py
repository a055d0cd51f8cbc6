"""C4 shape at test size: a batch of uneven alkane chains and rings
(workloads.alkane_batch), one context per molecule, cycles issued
concurrently (publicrelease_2020_b200.batch).  Each molecule's result equals
its own serial cycle bit for bit, and the smallest molecules match the FP64
oracle at the parity tolerances of tests/test_parity_gpu.py (LDA)."""
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


def test_concurrent_batch_equals_serial_cycles(batch):
    systems, b = batch
    b.cycle()                       # first cycle: buffers allocated
    t0 = time.perf_counter()
    par = b.cycle()
    t1 = time.perf_counter()
    ser = b.cycle_serial()
    t2 = time.perf_counter()
    print(f"batch of {len(systems)}: concurrent {t1 - t0:.3f} s, serial {t2 - t1:.3f} s")
    for s, p, q in zip(systems, par, ser):
        assert p["esic"] == q["esic"], s.name
        for k in ("results", "sic", "debdax", "cfrm"):
            assert np.array_equal(p[k], q[k]), (s.name, k)


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
