"""Many molecules of uneven size in one batch on one GPU.

Each molecule has its own context (geometry, orbitals, FODs, device buffers,
CUDA stream).  Batch.cycle runs one SIC cycle of every molecule through
flosic_sic_batch_cycle: each molecule's FO construction, FO values, pair
coefficients and POISSON1 call set-up on its own stream, then the Coulomb
potentials of all FOs of all molecules and both spins in two persistent
launches over one list of (molecule-spin, 128-point tile, FO block) items,
then each molecule's XC, energies, SIC matrix and forces.  This is the B200
form of the reference's orbital-parallel GROUP mode (global_call.F90:113-160),
where MPI groups take the FOs of a molecule; here the persistent CTAs take
tiles of every molecule.  Batch.autotune times the FO block widths (32, 64 or
128 FOs per item) on the batch itself and keeps the fastest.

Batch.cycle_streams is the earlier form kept for comparison: every molecule's
own flosic_sic_cycle issued from a pool of host threads, so the molecules'
kernels overlap on their streams."""
from __future__ import annotations

import time
from concurrent.futures import ThreadPoolExecutor

from . import sic


class Batch:
    """Contexts for a list of workloads.System on one device."""

    def __init__(self, systems, device=0, precision="fp64", workers=None):
        self.systems = list(systems)
        self.ctxs = []
        self.wm = 0  # FO block of the batched launch: 0 = from the largest FO count
        try:
            for s in self.systems:   # context creation (device set-up) stays serial
                c = sic.open_system(s, device)
                c.set_precision(precision)
                self.ctxs.append(c)
        except Exception:
            self.close()
            raise
        self.workers = workers or min(32, max(1, len(self.ctxs)))

    def cycle(self):
        """One SIC cycle of every molecule (flosic_sic_batch_cycle); a list of
        outputs shaped as FlosicSIC.cycle's."""
        return sic.batch_cycle(self.ctxs, self.wm)

    def autotune(self, reps=2, widths=(1, 2, 4)):
        """Time one batch cycle at each FO block width (32, 64, 128 FOs per
        item; the best of `reps` after one untimed run) and keep the fastest.
        The widths regroup FOs into items without changing any operation or its
        order, so the results do not depend on the choice.  Returns
        (width in FOs, {width: seconds})."""
        import torch
        times = {}
        for wm in widths:
            self.wm = wm
            self.cycle()
            best = float("inf")
            for _ in range(reps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                self.cycle()
                torch.cuda.synchronize()
                best = min(best, time.perf_counter() - t0)
            times[32 * wm] = best
        best_w = min(times, key=times.get)
        self.wm = best_w // 32
        return best_w, times

    def cycle_streams(self):
        """Every molecule's own flosic_sic_cycle from a pool of host threads."""
        with ThreadPoolExecutor(self.workers) as ex:
            return list(ex.map(lambda c: c.cycle(), self.ctxs))

    def cycle_serial(self):
        """The same cycles one molecule after another (reference for timing)."""
        return [c.cycle() for c in self.ctxs]

    def close(self):
        for c in self.ctxs:
            c.close()
        self.ctxs = []
