"""Generates tests/golden/c60_scan_results.npz: the FP64 oracle's RESULTS(1:13)
for the first two FOs of each spin of the C60 SCAN system at test size
(publicrelease_2020_b200.workloads.c60(nrad=4): 60 atoms, 900 functions,
180+180 FOs, 30,912 mesh points).  The oracle needs about two minutes of CPU
for these four FOs, too long to rerun with every GPU test, so its output is
committed; the GPU test regenerates the system (seeded) and compares.

    python tests/golden/make_c60_scan_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from publicrelease_2020_b200 import workloads as W  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c60_scan_results.npz")
NFO = 2

if __name__ == "__main__":
    sysm = W.c60(nrad=4)
    r = O.Oracle(sysm).sic_cycle(nthreads=os.cpu_count() or 1, fo_limit=NFO)
    np.savez(OUT, results=r["results"][:, :NFO], nmsh=sysm.nmsh, nbasis=sysm.nbasis,
             esic_partial=np.sum(r["results"][:, :NFO, 8]))
    print(OUT, r["results"][:, :NFO, 8])
