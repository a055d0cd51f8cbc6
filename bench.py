#!/usr/bin/env python
"""Benchmark: seconds per FLO-SIC SCF cycle (all FOs + FOD forces) on B200.

A step is one SIC block of an SCF iteration (main.F:577-759): FO construction,
APOTNL_SIC for every FO (basis values, Gaussian-pair Coulomb potential, XC),
the SIC matrix and the FOD forces, through the C ABI (flosic_sic_cycle).

Workload (N=1): the synthetic kernel shape -- 40 atoms in a 12 A cube, 512
contracted s/p/d functions (3 primitives each, exponents log-uniform in
[0.05, 1e4]), 1,000,000 mesh points, 128 FOs, PBE -- generated from a seed
(there is no dataset).  Multi-GPU (torchrun, NCCL): the same system's mesh
points are split into N shards, one per rank (flosic_sic_set_shard); a step
is one cycle with the one exchange of the path, an in-place NCCL all-reduce of
the packed partial sums (SIC matrix, APOTNL_SIC mesh sums) on the GPU, then
the combine on every rank -- strong scaling; value = max-over-ranks time of
one cycle.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s per FLO-SIC SCF cycle (all FOs + FOD forces), mixed vs FP64, |ΔE_SIC|≤10µHa"
COULOMB_FLOPS_NEAR = 92.0    # per near (pair, point, FO): 46 polynomial coefficients x Boys-monomial terms
COULOMB_FLOPS_TERM = 2.0     # per multipole term kept by the skip rule in a far (call, point, FO) evaluation
# DRAM bytes of the two Coulomb kernels per tile of 128 points on the C2 shape:
# ncu dram__bytes_read.sum + dram__bytes_write.sum on 296 tiles (k_coulomb_shared
# 7.951 GB + 0.041 GB, k_coulomb_perfo 1.828 GB + 0.179 GB); the traffic is
# re-reads of the per-call A operands, proportional to the tile count.
COULOMB_DRAM_BYTES_PER_TILE = (7.951e9 + 0.041e9 + 1.828e9 + 0.179e9) / 296
# (the Boys values, monomials and harmonics depend on geometry only and are
# formed once per (pair or call, point); the per-FO work is the contraction)


def workload(name):
    from publicrelease_2020_b200 import workloads as W
    if name == "c2":
        return W.synthetic(natoms=40, nbasis=512, nmsh=1_000_000, nfo=128, seed=1), \
            dict(workload="synthetic C2: 40 atoms, 512 s/p/d functions (3 prims), 1e6 mesh points, 128 FOs, PBE",
                 atoms=40, nbasis=512, nmsh=1_000_000, nfo=128, functional="GGA-PBE*GGA-PBE", nspn=1)
    if name == "c2half":
        return W.synthetic(natoms=40, nbasis=512, nmsh=250_000, nfo=128, seed=1), \
            dict(workload="synthetic C2 shape on a 2.5e5-point mesh", atoms=40, nbasis=512, nmsh=250_000, nfo=128,
                 functional="GGA-PBE*GGA-PBE", nspn=1)
    if name == "c2tiny":
        return W.synthetic(natoms=40, nbasis=512, nmsh=37_888, nfo=128, seed=1), \
            dict(workload="synthetic C2 shape on a 37888-point mesh: 296 tiles, two waves of 148 CTAs "
                          "(profiling case)", atoms=40, nbasis=512, nmsh=37_888, nfo=128,
                 functional="GGA-PBE*GGA-PBE", nspn=1)
    if name == "c2prof":
        return W.synthetic(natoms=10, nbasis=128, nmsh=250_000, nfo=64, box_ang=7.56, seed=1), \
            dict(workload="C2 density of atoms and points in a 7.56 A box: 10 atoms, 128 functions, 2.5e5 points, "
                          "64 FOs (profiling case)", atoms=10, nbasis=128, nmsh=250_000, nfo=64,
                 functional="GGA-PBE*GGA-PBE", nspn=1)
    if name == "c1":
        s = W.water(seed=0, nrad=60, basis="default")
        return s, dict(workload=f"C1 water LDA-PW91, default NRLMOL basis ({s.nbasis} functions), 5+5 FODs, "
                                f"{s.nmsh}-point atom-centred mesh", atoms=3, nbasis=s.nbasis, nmsh=s.nmsh, nfo=5,
                       functional="LDA-PW91*LDA-PW91", nspn=2)
    if name == "c3":
        s = W.benzene(seed=3, nrad=228, basis="default")
        return s, dict(workload=f"benzene LDA-PW91, 21+21 FODs, default NRLMOL basis ({s.nbasis} functions), "
                                f"{s.nmsh} mesh points",
                       atoms=12, nbasis=s.nbasis, nmsh=s.nmsh, nfo=21, functional="LDA-PW91*LDA-PW91", nspn=2)
    if name == "c5":
        s = W.c60(seed=4, nrad=40)
        return s, dict(workload=f"C60 SCAN, 180+180 FODs, {s.nbasis} functions, {s.nmsh} mesh points "
                                "(a tenth of the 3e6-point C60 mesh)",
                       atoms=60, nbasis=s.nbasis, nmsh=s.nmsh, nfo=180, functional="MGGA-SCAN*MGGA-SCAN", nspn=2)
    if name == "c5prof":
        s = W.c60(seed=4, nrad=8)
        return s, dict(workload=f"C60 SCAN, 180+180 FODs, {s.nbasis} functions, {s.nmsh} mesh points "
                                "(profiling case: about 480 tiles)",
                       atoms=60, nbasis=s.nbasis, nmsh=s.nmsh, nfo=180, functional="MGGA-SCAN*MGGA-SCAN", nspn=2)
    if name == "water":
        s = W.water(seed=0, nrad=40)
        return s, dict(workload="water LDA-PW91, 5+5 FODs", atoms=3, nbasis=s.nbasis, nmsh=s.nmsh, nfo=5,
                       functional="LDA-PW91*LDA-PW91", nspn=2)
    if name == "small":
        s = W.small_synthetic(seed=5, natoms=6, nbasis=60, nmsh=40000, nfo=12)
        return s, dict(workload="small synthetic", atoms=6, nbasis=60, nmsh=40000, nfo=12,
                       functional="GGA-PBE*GGA-PBE", nspn=1)
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for n, v in zip(names, r[3:7]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except Exception:
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_peak_tflops(torch):
    """Measured FP64 throughput of cuBLAS DGEMM on this GPU (roofline denominator
    for the FP64 Coulomb kernel; MEASURED_PEAKS.json carries no FP64 figure)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(5):
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def tf32_peak_tflops():
    """Dense TF32 tensor rate for the roofline of the tcgen05 TF32 kernel: half
    the bf16 burst rate the driver measured on this pool (MEASURED_PEAKS.json),
    as kind::tf32 issues half the MACs of kind::f16 per cycle; None without it."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]) / 2.0
    except (OSError, KeyError, ValueError):
        return None


def cpu_baseline(sysm, threads, reps=3):
    """The oracle (the reference algorithm restated in C++) timed on the host
    cores on a bounded sample, scaled to one full SCF cycle.

    Sample: every m-th mesh point (about 20,000 points) and as many FOs as
    threads, one FO per thread.  FOs are independent, so the FO count scales
    exactly.  The mesh does not scale by itself: POISSON1's near/far choice
    (poisson1.f:569-583) weighs point counts against a fixed 146-point sphere,
    so the sample weighs each of its points as m (set_count_scale) to make the
    full mesh's choices, and the work that does not depend on the points (pair
    coefficients, call set-up, moments) is timed separately on a 128-point
    sample with the same weighting and not scaled by m:
        T = F * (t0 + (t_m - t0) * N / n_m),   F = all FOs / sampled FOs.
    Each time is the best of `reps` runs (the host may be shared)."""
    from oracle import oracle as O
    import copy

    def sample(stride):
        sub = copy.copy(sysm)
        sub.rmsh = np.ascontiguousarray(sysm.rmsh[::stride])
        sub.wmsh = np.ascontiguousarray(sysm.wmsh[::stride] * stride)
        return sub

    nf = max(sysm.nfrm)
    nrun = min(nf, max(1, threads))
    fo_limit = nrun if nrun < nf else 0

    def timed(sub):
        orc = O.Oracle(sub)
        orc.set_count_scale(sysm.nmsh / sub.nmsh)
        best = 1e30
        for _ in range(reps):
            t0 = time.perf_counter()
            orc.sic_cycle(nthreads=threads, fo_limit=fo_limit)
            best = min(best, time.perf_counter() - t0)
        return best

    big, small = sample(max(1, sysm.nmsh // 20000)), sample(max(1, sysm.nmsh // 128))
    t_m, t_0 = timed(big), timed(small)
    per_point = max(t_m - t_0, 0.0) / big.nmsh
    nfo_total = sum(sysm.nfrm)
    fos = nrun * sysm.nspn if fo_limit else nfo_total
    value = (t_0 + per_point * sysm.nmsh) * nfo_total / fos
    return value, dict(points=big.nmsh, points0=small.nmsh, fos=fos, seconds=t_m, seconds0=t_0, reps=reps)


def sample_text(sysm, sample):
    return (f"oracle (reference algorithm restated in C++) on {sample['fos']} FOs: best of {sample['reps']} runs on "
            f"{sample['points']} of {sysm.nmsh} mesh points ({sample['seconds']:.2f} s) minus the point-independent "
            f"set-up timed on {sample['points0']} points ({sample['seconds0']:.2f} s), points weighted by the mesh "
            f"ratio in the near/far cost model, scaled to the full mesh and all FOs")


def run_reference(args, rank, world):
    if rank != 0:
        return
    sysm, cfg = workload(args.workload)
    threads = os.cpu_count() or 1
    vals = []
    sample = None
    for i in range(args.warmup + args.steps):
        v, sample = cpu_baseline(sysm, threads)
        if i >= args.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    cfg["parallelism"] = "host threads"
    cfg["fo_density"] = "pairs"  # the reference's own route (poisson1.f), which the CPU port follows
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port",
                         "sample": sample_text(sysm, sample)},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    from publicrelease_2020_b200 import sic as S

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    sysm, cfg = workload(args.workload)
    ctx = S.FlosicSIC(local_rank)
    if world > 1:
        ctx.set_shard(rank, world)
    ctx.set_geometry(sysm)
    ctx.set_orbitals(sysm.psi, sysm.nwfs, sysm.fods)
    ctx.set_density_mode(args.density)
    cfg["fo_density"] = args.density
    ld = ctx.ld
    if world > 1:
        from publicrelease_2020_b200.shard import sharded_cycle

        def step(out):
            return sharded_cycle(ctx, device=f"cuda:{local_rank}")
    else:
        def step(out):
            return ctx.cycle(out)

    def new_out():
        return dict(results=np.zeros(2 * ld * 13), sic=np.zeros(2 * ld * ld), debdax=np.zeros(2 * ld * 3),
                    cfrm=np.zeros(2 * ld * 3), esic=np.zeros(1))

    def barrier():
        if dist is not None:
            dist.barrier()

    tuned = {}

    def timed(mode, clk_sampler):
        """W warm-up and K timed SIC cycles in one precision; inputs resident."""
        ctx.set_precision(mode)
        if not args.no_autotune:
            width, ms = ctx.autotune(reps=1)
            tuned[mode] = {"perfo_fo_slots": width, "ms": {str(k): round(v, 3) for k, v in ms.items()}}
        out = new_out()
        for _ in range(args.warmup):
            step(out)
        acc = dict(coul_ms=0.0, near=0, far=0, terms=0, launches=0, stage=np.zeros(7),
                   kern={"shared": np.zeros(4), "perfo": np.zeros(4)})
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with clk_sampler as clk:
            e0.record()
            for _ in range(args.steps):
                r = step(out)
                st = ctx.stats()
                acc["coul_ms"] += st["stage_ms"][3]
                acc["near"] += st["near_evals"]
                acc["far"] += st["far_evals"]
                acc["terms"] += st["far_terms"]
                acc["launches"] += st["launches"]
                acc["stage"] += st["stage_ms"]
                for k, v in ctx.kernel_stats().items():
                    acc["kern"][k] += np.array(v, dtype=np.float64)
            e1.record()
            torch.cuda.synchronize()
            barrier()
        res = {k: np.array(v, copy=True) for k, v in r.items() if k != "esic"}
        res["esic"] = r["esic"]
        return e0.elapsed_time(e1), acc, res, clk.summary()

    modes = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    runs = {m: timed(m, ClockSampler(local_rank)) for m in modes}
    errors = None
    headline = modes[-1]
    if "fp64" in runs and "mixed" in runs:
        a, b = runs["fp64"][2], runs["mixed"][2]
        n = [sysm.nfrm[s] for s in range(sysm.nspn)]
        dsic = max(np.abs(a["sic"][s][:n[s], :n[s]] - b["sic"][s][:n[s], :n[s]]).max() for s in range(sysm.nspn))
        msic = max(np.abs(a["sic"][s][:n[s], :n[s]]).max() for s in range(sysm.nspn))
        errors = {"d_esic_ha": abs(a["esic"] - b["esic"]),
                  "max_d_esic_per_fo_ha": max(np.abs(a["results"][s][:n[s], 8] - b["results"][s][:n[s], 8]).max()
                                              for s in range(sysm.nspn)),
                  "max_d_sic_matrix_rel": dsic / msic,
                  "max_d_fod_force_ha_bohr": max(np.abs(a["debdax"][s][:n[s]] - b["debdax"][s][:n[s]]).max()
                                                 for s in range(sysm.nspn))}
        errors["gate_esic_1e-5_ha"] = bool(errors["d_esic_ha"] <= 1e-5)
        errors["gate_force_1e-4_ha_bohr"] = bool(errors["max_d_fod_force_ha_bohr"] <= 1e-4)
        if not (errors["gate_esic_1e-5_ha"] and errors["gate_force_1e-4_ha_bohr"]):
            headline = "fp64"
    t_ms, st_acc, r, clocks = runs[headline]
    # e2e: host buffers through the C ABI (KS orbitals + FODs in, results out), headline precision
    ctx.set_precision(headline)
    out = new_out()
    psi = np.ascontiguousarray(sysm.psi)
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        ctx.set_orbitals(psi, sysm.nwfs, sysm.fods)
        step(out)
    f1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = f0.elapsed_time(f1)
    h2d = psi.nbytes + 8 * 3 * ld * 2
    d2h = sum(v.nbytes for v in out.values())
    times = {m: runs[m][0] for m in runs}
    if dist is not None:
        keys = sorted(times)
        t = torch.tensor([times[k] for k in keys] + [e2e_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        times = {k: float(t[i]) for i, k in enumerate(keys)}
        e2e_ms = float(t[-1])
        t_ms = times[headline]
    ctx_stats = ctx.stats()
    ctx.close()
    if rank != 0:
        return
    per_step_s = t_ms / 1e3 / args.steps
    value = per_step_s
    coul_s = st_acc["coul_ms"] / 1e3 / args.steps
    # the work counters are the whole system's (summed over the shards); the
    # roofline is per GPU: this rank's Coulomb stage against its share
    flops = (st_acc["near"] * COULOMB_FLOPS_NEAR + st_acc["terms"] * COULOMB_FLOPS_TERM) / args.steps / world
    peak = fp64_peak_tflops(torch)
    achieved = flops / coul_s / 1e12 if coul_s > 0 else 0.0
    # per kernel: the counted work of each Coulomb kernel over its own event-timed
    # span, against the peak of the tensor path it runs on
    kernels = {}
    for k, (ms, near, far, terms) in st_acc["kern"].items():
        if ms <= 0 or (near == 0 and terms == 0):
            continue
        kflops = (near * COULOMB_FLOPS_NEAR + terms * COULOMB_FLOPS_TERM) / args.steps / world
        kach = kflops / (ms / 1e3 / args.steps) / 1e12
        if k == "shared" and headline == "mixed":
            tf32 = tf32_peak_tflops()
            kernels["k_coulomb_shared_tc"] = {
                "achieved": kach, "ms_per_cycle": ms / args.steps, "unit": "TFLOP/s",
                "peak": tf32 / 3 if tf32 else None, "frac": kach / (tf32 / 3) if tf32 else None,
                "peak_kind": "tcgen05 kind::tf32 dense rate (half the measured bf16 burst rate in "
                             "MEASURED_PEAKS.json) / 3: each counted product runs as three TF32 products"}
        else:
            kernels["k_coulomb_shared" if k == "shared" else "k_coulomb_perfo"] = {
                "achieved": kach, "ms_per_cycle": ms / args.steps, "unit": "TFLOP/s", "peak": peak,
                "frac": kach / peak if peak else None, "peak_kind": "FP64 DMMA (cuBLAS DGEMM measured in this run)"}
    ntiles = (cfg["nmsh"] + 127) // 128
    traffic = COULOMB_DRAM_BYTES_PER_TILE * ntiles if args.workload in ("c2", "c2half", "c2tiny") else None
    cfg.update(parallelism=(f"mesh shards x{world}, NCCL all-reduce of the partial sums" if world > 1
                            else "single GPU"), l2="working set >> L2 (126 MB)",
               npairs=ctx_stats["npairs"], ncalls=ctx_stats["ncalls"], precision=headline,
               autotune=tuned or "off")
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step_s * 1e3, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64" if headline == "fp64" else "f32+f64",
        "data": "synthetic (seeded)", "config": cfg,
        "e2e": {"value": e2e_ms / 1e3 / args.steps, "unit": "s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(st_acc["launches"]),
        "roofline": {"bound": "tensor", "kernel": "k_coulomb_shared + k_coulomb_perfo", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "traffic": traffic, "traffic_note": "ncu DRAM bytes of both kernels on the 296-tile C2 "
                                                         "shape, scaled by tile count",
                     "peak_kind": "FP64 cuBLAS DGEMM measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                     "work": f"{st_acc['near'] / args.steps:.4g} near (pair,point,FO) x {COULOMB_FLOPS_NEAR:.0f} + "
                             f"{st_acc['terms'] / args.steps:.4g} kept multipole terms x {COULOMB_FLOPS_TERM:.0f} flops "
                             f"({st_acc['far'] / args.steps:.4g} far (call,point,FO) evaluations)",
                     "kernels": kernels},
        "stage_ms": {k: round(float(v) / args.steps, 3) for k, v in
                     zip(["fo", "orbitals", "coul_setup", "coul_eval", "xc", "sicmat", "forces"], st_acc["stage"])},
        "esic": r["esic"],
        "clocks": clocks,
    }
    if len(runs) > 1:
        line["precision"] = {
            "headline": headline,
            "s_per_cycle": {m: times[m] / 1e3 / args.steps for m in runs},
            "stage_ms": {m: {k: round(float(v) / args.steps, 3) for k, v in
                             zip(["fo", "orbitals", "coul_setup", "coul_eval", "xc", "sicmat", "forces"],
                                 runs[m][1]["stage"])} for m in runs},
            "speedup_mixed_vs_fp64": times["fp64"] / times["mixed"],
            "mixed_vs_fp64_errors": errors,
            "clocks": {m: runs[m][3] for m in runs},
        }
    if world == 1 and not args.no_cpu_baseline:
        cb, sample = cpu_baseline(sysm, os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": cb, "unit": "s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": sample_text(sysm, sample)}
    print(json.dumps(line), flush=True)


def run_batch(args, rank, world, local_rank):
    """C4: 64 alkane-like chains and rings of uneven size in one batch on one
    GPU (batch.Batch): the Coulomb potentials of all FOs of all molecules in
    two persistent launches (flosic_sic_batch_cycle), FO block width chosen by
    the batch autotuner.  A step is one SIC cycle of every molecule; with N
    GPUs the molecules are dealt round-robin to the ranks (independent objects,
    no collective) and the step time is the maximum over ranks.  The earlier
    form (every molecule's own cycle from host threads, overlapping on their
    streams) is timed beside it for comparison."""
    import torch
    from publicrelease_2020_b200 import batch as B
    from publicrelease_2020_b200 import workloads as W

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    systems = W.alkane_batch(64)
    mine = systems[rank::world]
    bt = B.Batch(mine, device=local_rank)

    def barrier():
        if dist is not None:
            dist.barrier()

    tuned = {}
    streams_s = {}

    def timed(mode, clk_sampler):
        for c in bt.ctxs:
            c.set_precision(mode)
        if not args.no_autotune:
            w, ts = bt.autotune(reps=1)
            tuned[mode] = {"fo_block": w, "s": {str(k): round(v, 4) for k, v in ts.items()}}
        for _ in range(args.warmup):
            bt.cycle()
        acc = dict(near=0, far=0, terms=0, launches=0)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with clk_sampler as clk:
            e0.record()
            for _ in range(args.steps):
                res = bt.cycle()
                for c in bt.ctxs:
                    st = c.stats()
                    acc["near"] += st["near_evals"]
                    acc["terms"] += st["far_terms"]
                    acc["far"] += st["far_evals"]
                    acc["launches"] += st["launches"]
            e1.record()
            torch.cuda.synchronize()
            barrier()
        # the per-molecule form beside it (not the headline)
        bt.cycle_streams()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record()
        for _ in range(args.steps):
            bt.cycle_streams()
        g1.record()
        torch.cuda.synchronize()
        streams_s[mode] = g0.elapsed_time(g1) / 1e3 / args.steps
        return e0.elapsed_time(e1), acc, res, clk.summary()

    modes = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    runs = {m: timed(m, ClockSampler(local_rank)) for m in modes}
    headline = modes[-1]
    errors = None
    if len(runs) == 2:
        de = max(abs(a["esic"] - b["esic"]) for a, b in zip(runs["fp64"][2], runs["mixed"][2]))
        df = max(float(np.abs(a["debdax"][s][:m.nfrm[s]] - b["debdax"][s][:m.nfrm[s]]).max())
                 for a, b, m in zip(runs["fp64"][2], runs["mixed"][2], mine) for s in range(m.nspn))
        errors = {"max_d_esic_ha": de, "max_d_fod_force_ha_bohr": df,
                  "gate_esic_1e-5_ha": bool(de <= 1e-5), "gate_force_1e-4_ha_bohr": bool(df <= 1e-4)}
        if not (errors["gate_esic_1e-5_ha"] and errors["gate_force_1e-4_ha_bohr"]):
            headline = "fp64"
    for c in bt.ctxs:
        c.set_precision(headline)
    psis = [np.ascontiguousarray(m.psi) for m in mine]
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        for c, m, psi in zip(bt.ctxs, mine, psis):
            c.set_orbitals(psi, m.nwfs, m.fods)
        bt.cycle()
    f1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = f0.elapsed_time(f1)
    h2d = sum(psi.nbytes + 8 * 3 * c.ld * 2 for c, psi in zip(bt.ctxs, psis))
    d2h = sum(8 * (2 * c.ld * 13 + 2 * c.ld * c.ld + 4 * c.ld * 3 + 1) for c in bt.ctxs)
    times = {m: runs[m][0] for m in runs}
    if dist is not None:
        keys = sorted(times)
        t = torch.tensor([times[k] for k in keys] + [e2e_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        times = {k: float(t[i]) for i, k in enumerate(keys)}
        e2e_ms = float(t[-1])
    bt.close()
    if rank != 0:
        return
    t_ms, acc, _, clocks = runs[headline]
    t_ms = times[headline]
    per_step_s = t_ms / 1e3 / args.steps
    flops = (acc["near"] * COULOMB_FLOPS_NEAR + acc["terms"] * COULOMB_FLOPS_TERM) / args.steps * world
    peak = fp64_peak_tflops(torch)
    achieved = flops / per_step_s / 1e12
    nb = [m.nbasis for m in systems]
    npt = [m.nmsh for m in systems]
    nfo = [max(m.nfrm) for m in systems]
    cfg = {"workload": f"C4 batch: 64 alkane-like chains and rings (seeds 100-163, 2-29 atoms), {min(nb)}-{max(nb)} "
                       f"functions, {min(npt)}-{max(npt)} mesh points ({sum(npt)} in all), {min(nfo)}-{max(nfo)} FOs "
                       "per spin, LDA-PW91, NSPN=2; the Coulomb potentials of all molecules in two persistent "
                       "launches",
           "molecules": len(systems), "parallelism": (f"molecules dealt to {world} GPUs" if world > 1 else "single GPU"),
           "l2": "working set >> L2 (126 MB)", "precision": headline, "autotune": tuned or "off",
           "per_molecule_streams_s_per_cycle": streams_s}
    line = {
        "metric": METRIC, "value": per_step_s, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step_s * 1e3, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64" if headline == "fp64" else "f32+f64",
        "data": "synthetic (seeded)", "config": cfg,
        "e2e": {"value": e2e_ms / 1e3 / args.steps, "unit": "s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(acc["launches"]),
        "roofline": {"bound": "tensor", "kernel": "k_coulomb_shared + k_coulomb_perfo (whole batch cycle as the "
                                                  "denominator: the molecules' stages overlap)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "traffic": None,
                     "peak_kind": "FP64 cuBLAS DGEMM measured in this run (MEASURED_PEAKS.json has no FP64 figure)"},
        "clocks": clocks,
    }
    if len(runs) > 1:
        line["precision"] = {"headline": headline, "s_per_cycle": {m: times[m] / 1e3 / args.steps for m in runs},
                             "speedup_mixed_vs_fp64": times["fp64"] / times["mixed"],
                             "mixed_vs_fp64_errors": errors, "clocks": {m: runs[m][3] for m in runs}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="time the FP64 path, the mixed path, or both (headline = mixed when it meets the "
                         "|dE_SIC| <= 1e-5 Ha and FOD-force <= 1e-4 Ha/bohr gates)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c2half", "c2tiny", "c2prof", "c3", "c4", "c5", "c5prof", "water",
                                                      "small"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--density", default="phi2", choices=["phi2", "pairs"],
                    help="FO density route of the SIC XC: phi^2 from the FO values (default) or the "
                         "reference's Gaussian-pair route at each Poisson call's near points")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the per-FO Coulomb kernel's default tile width instead of timing the candidates")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.workload == "c4":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the CPU arm times single systems, "
                                                                      "not the C4 batch"}), flush=True)
            return
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.workload == "c4":
            run_batch(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
