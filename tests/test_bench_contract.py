"""CPU check of bench.py's output line: the keys and units the benchmark
contract asks for, for a single system (run_ours) and for the batch of
molecules (run_batch).  The library context, CUDA events and the clock
sampler are replaced by stand-ins that return fixed timings, so this tests
the bookkeeping (per-step time, e2e bytes, roofline fields, precision gates),
not the GPU; the GPU numbers come from running bench.py on a B200."""
import json
import types

import numpy as np
import pytest

import bench
from publicrelease_2020_b200 import batch as B
from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

STEP_MS = 12.0


class _Ctx:
    """Stand-in for sic.FlosicSIC: fixed results, a 1e-7 shift in mixed mode."""

    def __init__(self, device=0, sysm=None):
        self.mode, self.ld, self.sysm = "fp64", 1, sysm
        if sysm is not None:
            self.ld = max(sysm.nfrm)

    def set_shard(self, *a):
        pass

    def set_geometry(self, sysm):
        self.sysm, self.ld = sysm, max(sysm.nfrm)

    def set_orbitals(self, *a):
        pass

    def set_precision(self, mode):
        self.mode = mode

    def set_density_mode(self, mode):
        self.density = mode

    def autotune(self, reps=1):
        return 32, {32: 1.0}

    def cycle(self, out=None):
        ld, e = self.ld, (1e-7 if self.mode == "mixed" else 0.0)
        return dict(results=np.zeros((2, ld, 13)), sic=np.ones((2, ld, ld)), debdax=np.full((2, ld, 3), e),
                    cfrm=np.zeros((2, ld, 3)), esic=1.0 + e)

    def stats(self):
        return dict(launches=7, stage_ms=np.full(7, 1.0), npairs=3, ncalls=2, near_evals=1000, far_evals=50,
                    far_terms=200)

    def kernel_stats(self):
        return {"shared": (0.6, 600, 30, 120), "perfo": (0.4, 400, 20, 80)}

    def close(self):
        pass


class _Batch:
    def __init__(self, systems, device=0):
        self.ctxs = [_Ctx(sysm=s) for s in systems]
        self.wm = 0

    def cycle(self):
        return [c.cycle() for c in self.ctxs]

    def cycle_streams(self):
        return [c.cycle() for c in self.ctxs]

    def autotune(self, reps=2):
        self.wm = 2
        return 64, {32: 0.3, 64: 0.2, 128: 0.25}

    def close(self):
        pass


class _Event:
    def __init__(self, **k):
        pass

    def record(self):
        pass

    def elapsed_time(self, other):
        return STEP_MS


class _Clocks:
    def __init__(self, index):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        pass

    def summary(self):
        return {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}


@pytest.fixture
def fakes(monkeypatch):
    import torch
    small = W.water(seed=0, nrad=6)
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a: None)
    monkeypatch.setattr(torch.cuda, "set_device", lambda *a: None)
    monkeypatch.setattr(bench, "ClockSampler", _Clocks)
    monkeypatch.setattr(bench, "fp64_peak_tflops", lambda t: 35.0)
    monkeypatch.setattr(bench, "workload", lambda name: (small, dict(workload="water test shape", nspn=2,
                                                                       nmsh=small.nmsh)))
    monkeypatch.setattr(S, "FlosicSIC", _Ctx)
    monkeypatch.setattr(B, "Batch", _Batch)
    monkeypatch.setattr(W, "alkane_batch", lambda n: [small, small])
    return small


def _check_line(line, steps):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "roofline", "clocks"):
        assert k in line, k
    assert line["metric"] == bench.METRIC and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["value"] == pytest.approx(STEP_MS / 1e3 / steps)
    assert "workload" in line["config"]
    e2e = line["e2e"]
    assert set(e2e) == {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"}
    assert e2e["h2d_bytes_per_step"] > 0 and e2e["d2h_bytes_per_step"] > 0
    r = line["roofline"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in r, k
    assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    assert line["precision"]["headline"] == "mixed"
    gates = line["precision"]["mixed_vs_fp64_errors"]
    assert gates["gate_esic_1e-5_ha"] and gates["gate_force_1e-4_ha_bohr"]


def test_single_system_line(fakes, capsys):
    args = types.SimpleNamespace(workload="water", steps=2, warmup=3, precision="both", no_autotune=False,
                                 no_cpu_baseline=True, density="phi2")
    bench.run_ours(args, 0, 1, 0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    _check_line(line, 2)
    assert line["config"]["autotune"]["mixed"]["perfo_fo_slots"] == 32
    assert line["config"]["fo_density"] == "phi2"
    assert line["gpu_launches"] == 2 * 7
    kern = line["roofline"]["kernels"]
    assert set(kern) == {"k_coulomb_shared_tc", "k_coulomb_perfo"}   # mixed headline: TF32 shared kernel
    per = kern["k_coulomb_perfo"]
    # perfo: 2 steps x (400 near x 92 + 80 terms x 2) flops over 2 x 0.4 ms
    assert per["achieved"] == pytest.approx((400 * 92 + 80 * 2) / 0.4e-3 / 1e12)
    assert per["frac"] == pytest.approx(per["achieved"] / per["peak"])


def test_batch_line(fakes, capsys):
    args = types.SimpleNamespace(workload="c4", steps=2, warmup=3, precision="both", no_autotune=False)
    bench.run_batch(args, 0, 1, 0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    _check_line(line, 2)
    assert line["config"]["molecules"] == 2
    assert line["gpu_launches"] == 2 * 2 * 7
    assert line["config"]["autotune"]["mixed"]["fo_block"] == 64
    assert set(line["config"]["per_molecule_streams_s_per_cycle"]) == {"fp64", "mixed"}
