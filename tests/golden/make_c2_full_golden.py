"""Generates tests/golden/c2_full_results.npz: the FP64 oracle's RESULTS(1:13)
and SIC-matrix columns of the first four FOs of the full-size synthetic C2
system (publicrelease_2020_b200.workloads.synthetic: 40 atoms, 512 functions,
1,000,000 mesh points, 128 FOs, PBE, NSPN=1).  SIC(j, l) needs only FO l's
potential, so the columns l = 1..4 come from the oracle's SICLAGM given those
four potentials (the other columns are left out).  The oracle needs tens of
CPU-minutes for this, far too long for a test, so its output is committed; the
GPU test regenerates the system (seeded) and compares.

    python tests/golden/make_c2_full_golden.py
"""
import os
import sys
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from publicrelease_2020_b200 import workloads as W  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_full_results.npz")
NFO = 4


def system():
    return W.synthetic(natoms=40, nbasis=512, nmsh=1_000_000, nfo=128, seed=1)


if __name__ == "__main__":
    sysm = system()
    orcs = [O.Oracle(sysm) for _ in range(NFO)]  # one oracle per thread (each call releases the GIL)
    with ThreadPoolExecutor(NFO) as ex:
        outs = list(ex.map(lambda k: orcs[k - 1].apotnl_sic(1, k), range(1, NFO + 1)))
    orc = orcs[0]
    results = np.stack([o["results"] for o in outs])
    pots = np.zeros((sysm.nfrm[0], sysm.nmsh))
    for k, o in enumerate(outs):
        pots[k] = o["pot"]
    lam = orc.siclagm(1, pots)
    # lam[l][j] = SIC(j, l): the first NFO columns
    np.savez(OUT, results=results, sic_cols=np.ascontiguousarray(lam[:NFO, : sysm.nfrm[0]]), nmsh=sysm.nmsh,
             nbasis=sysm.nbasis, nfo=sysm.nfrm[0])
    print(OUT, results[:, 8])
