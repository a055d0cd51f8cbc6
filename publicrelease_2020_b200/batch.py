"""Many molecules of uneven size in one batch on one GPU.

Each molecule has its own context (its own CUDA stream, cuBLAS/cuSOLVER
handles and device buffers); a cycle of the batch issues every molecule's SIC
cycle from a pool of host threads, so the kernels of different molecules
overlap on the GPU instead of running one molecule after another (ctypes
releases the interpreter lock during each library call).  After the first
cycle no context allocates device memory, so the molecules' streams do not
synchronise each other.  Results are those of the molecules' own cycles,
bit for bit: every context computes in its own deterministic order."""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

from . import sic


class Batch:
    """Contexts for a list of workloads.System on one device."""

    def __init__(self, systems, device=0, precision="fp64", workers=None):
        self.systems = list(systems)
        self.ctxs = []
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
        """One SIC cycle of every molecule; a list of flosic_sic_cycle outputs."""
        with ThreadPoolExecutor(self.workers) as ex:
            return list(ex.map(lambda c: c.cycle(), self.ctxs))

    def cycle_serial(self):
        """The same cycles one molecule after another (reference for timing)."""
        return [c.cycle() for c in self.ctxs]

    def close(self):
        for c in self.ctxs:
            c.close()
        self.ctxs = []
