"""Benchmark of the matrix-profile self-join on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (one GPU): c2 -- a random walk of n = 1,048,576 samples
(seed 1), window m = 256, exclusion zone m/4, every diagonal of the distance
matrix (5.49e11 cells).  One step = one complete self-join.  Metric: cells/s
of the FP32 recurrence re-anchored in FP64 every K = 1024 steps, reported
beside the plain FP64 GPU kernel on the same input and the FP32 form's
maximum relative distance error against it.

Timing: W untimed warm-up steps, then K steps, each bracketed by CUDA events
on the stream the library launches on; an L2 flush (256 MB write) runs between
steps outside the events; barrier + device synchronisation around the loop;
the maximum over ranks is reported.  With N > 1 the diagonals are split into
2N partitions, rank r taking partitions r and 2N-1-r (the reference's
scrimp_triv_par balance rule) in one mp_selfjoin_ranges call, and the partial
profiles are merged with NCCL MIN all-reduces of packed keys (one for the
FP32 form, two for the FP64 form; shard.allreduce_profiles).

--impl reference times the reference's own CPU code (oracle/_ref, built from
its unchanged sources; else the C restatement) on all host cores, each step a
bounded diagonal sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MP cells/s vs plain FP64 GPU kernel at ≤1e-4 rel. error; p50/p99 solve latency"
FLOP_PER_CELL = 8  # 2 FMA for the dot-product update, 1 FMA + 2 MUL for the score


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_model() -> str:
    """The host CPU's model name (from /proc/cpuinfo), or the platform's."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.lower().startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or platform.machine()


def sample_range(n: int, m: int, target_cells: float):
    """Diagonal range [excl+1, hi) holding about target_cells cells."""
    PL, lo = n - m + 1, m // 4 + 1
    hi, cells = lo, 0.0
    step = max(1, (PL - lo) // 4096)
    while hi < PL and cells < target_cells:
        h2 = min(PL, hi + step)
        cells += sum(PL - d for d in range(hi, h2))
        hi = h2
    return lo, hi, cells


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.devices = [device] if isinstance(device, int) else list(device)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", ",".join(str(d) for d in self.devices)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


SERIES_KIND = {
    "c3": "random walk with 32 sine motifs and 16 constant stretches at the walk's level,",
    "c3z": "random walk with 32 sine motifs and 16 constant stretches at level 0,",
}


def read_ncu_traffic(kernel: str):
    """dram bytes per launch recorded in profiles/ (from one ncu capture)."""
    path = os.path.join(ROOT, "profiles", f"{kernel}.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch_full:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def cpu_reference_run(x, m, target_seconds: float, threads: int):
    """Times the reference CPU path on `threads` host threads over a diagonal
    sample of about target_seconds.  Returns (cells, seconds, kind, sample)."""
    from oracle.oracle import Oracle, RefOracle, build
    n = x.size
    kind = "reference" if RefOracle.available("ieee") else "port"
    per_core = 1.0e9 if kind == "reference" else 4.0e8  # cells/s/core, sizing only
    lo, hi, cells = sample_range(n, m, per_core * threads * target_seconds)
    if kind == "reference":
        ref = RefOracle("fast")  # the reference's release flags
        _, _, sec = ref.triv_par_threads(x, m, lo, hi, threads)
    else:
        if not os.path.exists(os.path.join(ROOT, "oracle", "libscrimp_oracle.so")):
            build(with_reference=False)
        t0 = time.perf_counter()
        Oracle().selfjoin(x, m, diag_lo=lo, diag_hi=hi, nthreads=threads)
        sec = time.perf_counter() - t0
    sample = (f"diagonals [{lo}, {hi}) of the same series: {cells:.3e} cells, "
              f"{threads} threads, scrimp_triv_par partitioning re-hosted on threads")
    return cells, sec, kind, sample


def parity_checks(ctx, workload, x, m, d2_64, idx_64, d2_32):
    """This run's GPU results against the reference, outside the timed region.

    - digest: SHA-256 of the FP64 form's squared distances (and indices) against
      the digests tests/golden/make_golden.py recorded from the reference's own
      code for this workload (c1, c2);
    - index_sample: for a seeded sample of windows, the reference's own score of
      the cell (window, chosen neighbour), recomputed on the host with the
      reference's per-cell arithmetic, gives exactly the FP64 form's squared
      distance (so the neighbour attains the profile value; a different index
      in the reference can only be an exact tie);
    - fp32_vs_fp64: the FP32 form's relative distance error against that FP64
      profile (the bound is 1e-4);
    - test_ascii: the FP64 form on the reference's own fixture
      (data_testing/test.ascii, m in {16, 64, 400}) against its golden profiles,
      bit for bit, indices by the same tie rule.
    """
    import hashlib

    import thesiscode_b200 as mp
    from oracle.oracle import Oracle
    golden = os.path.join(ROOT, "tests", "golden")
    orc = Oracle()
    out = {}
    digests = json.load(open(os.path.join(golden, "digests.json")))
    if workload in digests:
        want = digests[workload]
        out["digest"] = {
            "workload": workload,
            "d2_sha256_match": hashlib.sha256(d2_64.tobytes()).hexdigest() == want["d2_sha256"],
            "idx_sha256_match": hashlib.sha256(idx_64.tobytes()).hexdigest() == want["idx_sha256"],
        }

    def neighbour_attains(xs, mm, d2, idx, wins):
        stats = orc.window_stats(xs, mm)
        valid = [i for i in wins if not (d2[i] == 2 * mm + 2 and idx[i] == 0)]
        if not valid:
            return 0, 0
        i = np.asarray(valid, dtype=np.int64)
        j = idx[i]
        s = orc.cell_scores(xs, mm, np.minimum(i, j), np.maximum(i, j), 500, stats=stats)
        return int(np.sum(2.0 * mm - 2.0 * s != d2[i])), len(valid)

    rng = np.random.default_rng(7)
    PL = x.size - m + 1
    wins = rng.choice(PL, size=min(256, PL), replace=False)
    bad, checked = neighbour_attains(x, m, d2_64, idx_64, wins)
    out["index_sample"] = {"windows": checked, "neighbour_not_attaining_value": bad}
    dt = np.sqrt(np.abs(d2_64))
    rel = np.abs(np.sqrt(np.abs(d2_32)) - dt) / dt
    out["fp32_vs_fp64"] = {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()),
                           "bound": 1e-4, "within": bool(rel.max() <= 1e-4)}
    ga = np.load(os.path.join(golden, "test_ascii.npz"))
    series = ga["series"]
    ta = {}
    for mm in (16, 64, 400):
        p = ctx.selfjoin(series, mm, precision=mp.FP64)
        diff = np.nonzero(p.index != ga[f"idx_m{mm}"])[0]
        ties = 0
        if diff.size:
            stats = orc.window_stats(series, mm)
            a, b = p.index[diff], ga[f"idx_m{mm}"][diff]
            sa = orc.cell_scores(series, mm, np.minimum(diff, a), np.maximum(diff, a), 500,
                                 stats=stats)
            sb = orc.cell_scores(series, mm, np.minimum(diff, b), np.maximum(diff, b), 500,
                                 stats=stats)
            da, db = np.sqrt(np.abs(2.0 * mm - 2.0 * sa)), np.sqrt(np.abs(2.0 * mm - 2.0 * sb))
            ties = int(np.sum((sa == sb) | (np.abs(da - db) <= 1e-9 * db)))
        ta[f"m{mm}"] = {"d2_bit_identical": bool(np.array_equal(p.dist2, ga[f"d2_m{mm}"])),
                        "index_differences": int(diff.size), "of_which_ties": ties}
    out["test_ascii"] = ta
    out["all_pass"] = bool(
        out.get("digest", {}).get("d2_sha256_match", True) and bad == 0
        and out["fp32_vs_fp64"]["within"]
        and all(v["d2_bit_identical"] and v["index_differences"] == v["of_which_ties"]
                for v in ta.values()))
    return out


def c3_sample(ctx, width: int, k: int):
    """Error of the FP32 and guarded forms against the FP64 form (the reference's
    arithmetic) on a diagonal sample of the stress series: c3 (n = 8,388,608,
    m = 1024, 32 planted sine motifs, 16 constant stretches at the walk's level)
    and c3z (the stretches at level 0), diagonals [m/4 + 1, m/4 + 1 + width).
    Per form: cells/s on the sample and the error figures of error_report
    (maximum far from the stretches and near them, windows whose FP64 value is
    itself inaccurate excluded)."""
    import thesiscode_b200 as mp
    from thesiscode_b200 import error_report as er
    out = {}
    for name in ("c3", "c3z"):
        x, m, segs, _ = er.load(name)
        lo = m // 4 + 1
        hi = lo + width
        cells = mp.cells(x.size, m, lo, hi)
        p64 = ctx.selfjoin(x, m, precision=mp.FP64, diag_lo=lo, diag_hi=hi)
        j64 = ctx.last_phase_ms()[1]
        rec = {"diagonals": [lo, hi], "cells": cells,
               "fp64_cells_per_s": cells / (j64 * 1e-3),
               "note": "a sample of few long diagonals: the FP64 form's bands (256 diagonals "
                       "each) fill under one wave of the GPU, so its rate here is not the full "
                       "join's; the FP32 form's tiles fill it"}
        # each form at its re-anchor interval: k for the FP32 form, the guarded
        # form's own default (512) for it
        for form, prec, kf in (("fp32", mp.FP32_REANCHOR, k), ("guarded", mp.FP32_GUARDED, 512)):
            p = ctx.selfjoin(x, m, precision=prec, reanchor_k=kf, diag_lo=lo, diag_hi=hi)
            j = ctx.last_phase_ms()[1]
            r = er.compare(x, m, segs, p64, p, name == "c3z", K=kf)
            rec[form] = {"reanchor_k": kf, "cells_per_s": cells / (j * 1e-3),
                         "max_rel_far_from_stretches": r["max_rel_far_from_stretches"],
                         "max_rel_near_stretches": r["max_rel_near_stretches"],
                         "mean_rel": r["mean_rel"], "reference_inaccurate": r["reference_inaccurate"]}
        out[name] = rec
    return out


def run_reference_arm(args, world):
    import thesiscode_b200.workloads as wl
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    x, m = wl.c2()
    threads = host_cores()
    vals = []
    for it in range(args.warmup + args.steps):
        cells, sec, kind, sample = cpu_reference_run(x, m, args.ref_seconds, threads)
        if it >= args.warmup:
            vals.append((cells, sec))
    cells = sum(c for c, _ in vals)
    sec = sum(s for _, s in vals)
    v = cells / sec
    import thesiscode_b200 as mp
    total = mp.cells(x.size, m)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "cells/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sec / len(vals), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "c2: random walk n=1,048,576 seed 1, m=256, excl=64; each step a "
                               "bounded diagonal sample (the longest diagonals) timed as a rate",
                   "n": int(x.size), "m": m, "cells_per_step": cells / len(vals),
                   "sample_fraction": cells / len(vals) / total,
                   "cpu_model": cpu_model(), "threads": threads,
                   "parallelism": "the reference's kernels.cpp (fast-math build) on host threads, "
                                  "scrimp_triv_par partitioning re-hosted on threads (no MPI)"},
        "cpu_baseline": {"value": v, "unit": "cells/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": v, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, world):
    import torch
    import torch.distributed as dist

    import thesiscode_b200 as mp
    import thesiscode_b200.workloads as wl

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.workload == "c1":
        x, m = wl.c1()
    elif args.workload in ("c3", "c3z"):
        # long stress series: motifs and constant stretches (at the walk's level, or 0)
        x, m, _ = wl.c3(zero_level=args.workload == "c3z")
    else:
        x, m = wl.c2()
    n = x.size
    from thesiscode_b200 import shard
    PL, excl = n - m + 1, m // 4
    mine = shard.rank_ranges(n, m, rank, world)
    cells_mine = sum(mp.cells(n, m, a, b) for a, b in mine)
    cells_total = mp.cells(n, m)

    ctx = mp.Context(local)
    ctx.set_phase_timing(True)
    stream = torch.cuda.Stream(device=dev)
    xd = torch.from_numpy(x).to(dev)
    d2 = torch.empty(PL, dtype=torch.float64, device=dev)
    ix = torch.empty(PL, dtype=torch.int64, device=dev)
    d2b = torch.empty_like(d2)
    ixb = torch.empty_like(ix)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def one_step(precision):
        # one call over this rank's diagonal partitions (one preparation, one
        # sync), then, with N > 1, the MIN all-reduce of packed keys
        ctx.selfjoin_ranges(xd, m, mine, precision=precision, reanchor_k=args.reanchor_k,
                            out=(d2, ix), stream=stream.cuda_stream)
        launches = ctx.last_launch_count
        join_ms = ctx.last_phase_ms()[1]
        if world > 1:
            with torch.cuda.stream(stream):
                md, mi = shard.allreduce_profiles(d2, ix, m, fp32_form=precision != mp.FP64)
                d2.copy_(md)
                ix.copy_(mi)
        return launches, join_ms

    def timed(precision, steps, warmup):
        for _ in range(warmup):
            one_step(precision)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        evs = []
        launches = 0
        join_ms = []
        with ClockSampler(local) as clk:
            for _ in range(steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                l, j = one_step(precision)
                e1.record(stream)
                evs.append((e0, e1))
                launches += l
                join_ms.append(j)
            torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        per = [a.elapsed_time(b) for a, b in evs]
        return per, launches, join_ms, clk.summary()

    # -- FP32 re-anchored form (headline) ------------------------------------
    per, launches, join_ms, clocks = timed(mp.FP32_REANCHOR, args.steps, args.warmup)
    total_ms = sum(per)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = cells_total * args.steps / (total_ms * 1e-3)
    fp32_d2 = d2.cpu().numpy().copy()
    fp32_idx = ix.cpu().numpy().copy()

    # -- plain FP64 GPU kernel on the same input ---------------------------------
    fsteps = max(1, min(args.steps, args.fp64_steps))
    per64, _, join64, _ = timed(mp.FP64, fsteps, 1)
    tot64 = sum(per64)
    if world > 1:
        t = torch.tensor([tot64], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot64 = float(t.item())
    value64 = cells_total * fsteps / (tot64 * 1e-3)
    fp64_d2 = d2.cpu().numpy().copy()
    fp64_idx = ix.cpu().numpy().copy()

    # -- end to end with pinned host buffers ----------------------------------------
    # N = 1: one mp_selfjoin call on host pointers (it copies in and out itself).
    # N > 1: every rank copies the series in, joins its diagonal partitions in
    # one call and merges through one MIN all-reduce (shard.distributed_selfjoin);
    # rank 0 reads the profile back.  Timed per rank with CUDA events, max over
    # ranks.
    xh = torch.from_numpy(x).pin_memory()
    oh = (torch.empty(PL, dtype=torch.float64).pin_memory(),
          torch.empty(PL, dtype=torch.int64).pin_memory())
    xdev = torch.empty(n, dtype=torch.float64, device=dev)
    parts = (torch.empty(PL, dtype=torch.float64, device=dev),
             torch.empty(PL, dtype=torch.int64, device=dev))

    def e2e_step():
        if world == 1:
            ctx.selfjoin(xh, m, precision=mp.FP32_REANCHOR, reanchor_k=args.reanchor_k, out=oh,
                         stream=stream.cuda_stream)
            return
        with torch.cuda.stream(stream):
            xdev.copy_(xh, non_blocking=True)

        def compute(ranges):
            d, i = parts
            ctx.selfjoin_ranges(xdev, m, ranges, precision=mp.FP32_REANCHOR,
                                reanchor_k=args.reanchor_k, out=(d, i), stream=stream.cuda_stream)
            return d, i

        with torch.cuda.stream(stream):
            md, mi = shard.distributed_selfjoin(compute, n, m, fp32_form=True)
            if rank == 0:
                oh[0].copy_(md, non_blocking=True)
                oh[1].copy_(mi, non_blocking=True)

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    lat = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(2.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        e2e_step()
        e1.record(stream)
        e1.synchronize()
        lat.append(e0.elapsed_time(e1))
    tot_e2e = sum(lat)
    if world > 1:
        t = torch.tensor([tot_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_e2e = float(t.item())
    # the FP64 form end to end: one mp_selfjoin call on pinned host buffers per step
    e2e64 = None
    if world == 1:
        ctx.selfjoin(xh, m, precision=mp.FP64, out=oh, stream=stream.cuda_stream)
        lat64 = []
        for _ in range(fsteps):
            with torch.cuda.stream(stream):
                flush.fill_(3.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.selfjoin(xh, m, precision=mp.FP64, out=oh, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            lat64.append(e0.elapsed_time(e1))
        e2e64 = {"value": cells_total * len(lat64) / (sum(lat64) * 1e-3), "unit": "cells/s",
                 "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 16 * PL,
                 "path": "mp_selfjoin (C ABI), FP64 form, pinned host input/outputs"}

    e2e = {"value": cells_total * len(lat) / (tot_e2e * 1e-3), "unit": "cells/s",
           "h2d_bytes_per_step": 8 * n * world, "d2h_bytes_per_step": 16 * PL,
           "path": "mp_selfjoin (C ABI) with pinned host input/outputs" if world == 1 else
           f"pinned host series to each of {world} GPUs, one mp_selfjoin_ranges call over the "
           "rank's two diagonal partitions, "
           "NCCL MIN all-reduce of packed keys (shard.distributed_selfjoin), profile to pinned host "
           "on rank 0"}

    # the FP64 form's phases on one more (untimed) call: preparation holds the
    # reference-order statistics and the first dot products of every diagonal
    phases64 = None
    if world == 1:
        ctx.selfjoin(xd, m, precision=mp.FP64, out=(d2b, ixb), stream=stream.cuda_stream)
        pp, pj, pf = ctx.last_phase_ms()
        phases64 = {"prep_ms": pp, "join_ms": pj, "finalize_ms": pf}

    if rank != 0:
        ctx.close()
        return

    # error of the FP32 form against the FP64 kernel (bit-identical to the reference)
    dt = np.sqrt(np.abs(fp64_d2))
    rel = np.abs(np.sqrt(np.abs(fp32_d2)) - dt) / dt
    err = {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()),
           "index_agreement": float(np.mean(fp32_idx == fp64_idx))}

    # roofline of the dominant kernel (the FP32 tile join)
    join_avg_ms = float(np.mean(join_ms)) if join_ms else float("nan")
    achieved = FLOP_PER_CELL * cells_mine / (join_avg_ms * 1e-3) / 1e12
    peaks = {}
    for which, name in ((0, "f32_ffma"), (1, "f32x2_ffma2"), (2, "f64_dfma")):
        try:
            peaks[name] = mp.measure_fma_peak(local, which) / 1e12
        except Exception:
            peaks[name] = None
    peak32 = max(v for v in (peaks["f32_ffma"], peaks["f32x2_ffma2"]) if v)
    traffic = read_ncu_traffic(f"fp32_join_kernel_{args.workload}")  # null without a capture
    roofline = {
        "bound": "fp32-fma-pipe (CUDA cores; no tensor-core or HBM bound)",
        "achieved": achieved, "peak": peak32, "unit": "TFLOP/s", "frac": achieved / peak32,
        "traffic": traffic, "kernel": "fp32_join_kernel<8, false>",
        "algorithmic_flops_per_launch": FLOP_PER_CELL * cells_mine,
        "kernel_ms": join_avg_ms,
        "peak_source": "measured in this run: independent-FMA-chain kernel (mp_measure_fma_peak), "
                       "max of FFMA and f32x2 FFMA2 rates; MEASURED_PEAKS.json has no CUDA-core "
                       "peak",
        "peaks_tflops": peaks,
    }
    join64 = float(np.mean(join64)) if join64 else float("nan")
    roof64 = FLOP_PER_CELL * cells_mine / (join64 * 1e-3) / 1e12

    line = {
        "metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{args.workload}: {SERIES_KIND.get(args.workload, 'random walk')} "
                               f"n={n:,}, m={m}, excl={excl}, all "
                               f"diagonals; FP32 recurrence re-anchored in FP64 every "
                               f"K={args.reanchor_k} steps",
                   "n": n, "m": m, "reanchor_k": args.reanchor_k, "cells": cells_total,
                   "l2": f"flushed between steps (256 MB write); working set "
                         f"~{(8 * n + 80 * PL) / 1e6:.0f} MB",
                   "parallelism": f"diagonal partitions x{2 * world}, NCCL MIN all-reduce merge"
                   if world > 1 else "single GPU"},
        "fp64_baseline": {"value": value64, "unit": "cells/s", "ms_per_step": tot64 / fsteps,
                          "kernel": "fp64_band_kernel (reference arithmetic, bit-identical)",
                          "roofline_frac_f64": roof64 / peaks["f64_dfma"] if peaks["f64_dfma"]
                          else None, "kernel_ms": join64, "phases": phases64, "e2e": e2e64},
        # the reference logs "(PL - excl)^2 / t" as its throughput (ScrimpVertBlocked
        # PERF_LOG); the same figure for this run, beside the true cell count
        "reference_log_metric": {"value": float(PL - excl) ** 2 / (total_ms / args.steps * 1e-3),
                                 "unit": "matrix entries/s, (PL - excl)^2 / t"},
        "speedup_vs_fp64": value / value64,
        "error_vs_fp64": err,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))}
        if lat else None,
        "roofline": roofline,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    line["e2e"] = e2e
    if world == 1 and not args.no_extras:
        # the batched (c4), serving (c5) and stress-series (c3) forms, summarised
        ctx.close()
        ctx = None
        torch.cuda.empty_cache()
        b = batch_measure(args.c4_count, 1, 1, 1)
        line["batch"] = {k: b[k] for k in ("value", "unit", "ms_per_step", "e2e", "config",
                                           "gpu_launches", "clocks")}
        srv = serving_measure(args.extra_rates, args.extra_serve_seconds, args.slots, 1)
        line["serving"] = [{k: r[k] for k in ("rate_hz", "duration_s", "requests", "completed",
                                              "rejected", "p50_ms", "p99_ms", "queue_p50_ms",
                                              "cells_per_s", "slots")} for r in srv]
        with mp.Context(local) as cctx:
            cctx.set_phase_timing(True)
            line["c3_sample"] = c3_sample(cctx, args.c3_width, args.reanchor_k)
        ctx = mp.Context(local)
    if world == 1 and not args.no_cpu_baseline:
        # the reference's CPU code: parity of this run's profiles, then its speed
        line["parity"] = parity_checks(ctx, args.workload, x, m, fp64_d2, fp64_idx, fp32_d2)
        threads = host_cores()
        cells, sec, kind, sample = cpu_reference_run(x, m, args.ref_seconds, threads)
        line["cpu_baseline"] = {"value": cells / sec, "unit": "cells/s", "cores": threads,
                                "kind": kind, "sample": sample, "cpu_model": cpu_model()}
        c1, s1, k1, smp1 = cpu_reference_run(x, m, min(3.0, args.ref_seconds), 1)
        line["cpu_baseline_1core"] = {"value": c1 / s1, "unit": "cells/s", "cores": 1, "kind": k1,
                                      "sample": smp1}
    print(json.dumps(line), flush=True)
    ctx.close()


def batch_measure(c4_count, gpus, steps, warmup):
    """Workload c4: FP32-input walks (lengths log-uniform in [2048, 262144], m in
    {64, 128, 256}, seed 3) solved by one persistent, graph-captured launch per
    step; tile widths from the autotuner table.  With gpus > 1 the series are
    split into groups of nearly equal cells (shard.balance_by_cost) and each GPU
    runs its group as its own batch (replicas, nothing exchanged); a step lasts
    until the slowest GPU is done.  Returns the measurement as a dict."""
    import threading

    import torch

    import thesiscode_b200 as mp
    import thesiscode_b200.workloads as wl
    from thesiscode_b200 import shard
    data = wl.c4(c4_count)
    lens = [x.size for x, _ in data]
    ms = [m for _, m in data]
    groups = shard.balance_by_cost([mp.cells(n, m) for n, m in zip(lens, ms)], max(1, gpus))
    reps = []  # (context, batch, stream, series) per GPU with work
    for d, g in enumerate(groups):
        if not g:
            continue
        ctx = mp.Context(d)
        b = mp.Batch(ctx, [lens[i] for i in g], [ms[i] for i in g], None, input_f32=True)
        st = torch.cuda.Stream(device=d)
        series = [data[i][0] for i in g]
        b.upload(series, st.cuda_stream)
        reps.append((ctx, b, st, series))
    for _ in range(warmup):
        for _, b, st, _ in reps:
            b.launch(st.cuda_stream)
    for _, _, st, _ in reps:
        st.synchronize()
    steps_ms = []
    with ClockSampler([d for d, g in enumerate(groups) if g]) as clk:
        for _ in range(steps):
            evs = []
            for _, b, st, _ in reps:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                b.launch(st.cuda_stream)
                e1.record(st)
                evs.append((e0, e1))
            for _, _, st, _ in reps:
                st.synchronize()
            steps_ms.append(max(a.elapsed_time(c) for a, c in evs))
    ms_step = float(np.mean(steps_ms))
    cells = sum(b.cells for _, b, _, _ in reps)
    # end to end through the public API: host series in, host profiles out,
    # into output arrays allocated once (as a serving loop would keep them);
    # one host thread per GPU
    outs = [b.outputs() for _, b, _, _ in reps]

    def run_all():
        ths = [threading.Thread(target=b.run, args=(series, st.cuda_stream), kwargs={"out": o})
               for (_, b, st, series), o in zip(reps, outs)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()

    for _ in range(max(1, warmup)):
        run_all()
    t0 = time.perf_counter()
    for _ in range(steps):
        run_all()
    e2e_s = (time.perf_counter() - t0) / steps
    launches = sum(b.launch_count for _, b, _, _ in reps)
    out = {"value": cells / (ms_step * 1e-3), "unit": "cells/s", "n_gpus": len(reps),
           "steps": steps, "warmup": warmup, "ms_per_step": ms_step, "dtype": "f32",
           "config": {"workload": f"c4: {len(data)} FP32 random walks, lengths log-uniform "
                                  f"[2048, 262144], m in {{64,128,256}}, seed 3",
                      "series": len(data), "samples": int(sum(lens)), "cells": cells,
                      "tiles": sum(b.tiles for _, b, _, _ in reps),
                      "launches_per_step": launches,
                      "parallelism": f"{len(reps)} replicas, series balanced by cells"},
           "e2e": {"value": cells / e2e_s, "unit": "cells/s",
                   "h2d_bytes_per_step": 4 * int(sum(lens)),
                   "d2h_bytes_per_step": 16 * int(sum(l - m + 1 for l, m in zip(lens, ms)))},
           "gpu_launches": launches * steps, "clocks": clk.summary()}
    for ctx, b, _, _ in reps:
        b.close()
        ctx.close()
    return out


def run_batch_workload(args):
    line = batch_measure(args.c4_count, args.gpus, args.steps, args.warmup)
    line = {"metric": "batched self-join cells/s (c4, one persistent graph-captured launch)",
            **line, "data": "synthetic", "scaling": "strong"}
    print(json.dumps(line), flush=True)


def serving_measure(rates, seconds, slots, gpus):
    """Workload c5: Poisson request streams at several rates against the
    continuous-batching server; p50/p99 latency and admitted cells/s per rate."""
    from thesiscode_b200.serve import run_stream
    out = []
    for rate in rates:
        # gpus > 1: one server per GPU, requests handed out in turn
        out.append(run_stream(rate, seconds, slots=slots, devices=list(range(max(1, gpus)))))
    return out


def run_serving_workload(args):
    for r in serving_measure(args.rates, args.serve_seconds, args.slots, args.gpus):
        r["metric"] = "serving p50/p99 solve latency (c5)"
        r["n_gpus"] = max(1, args.gpus)
        print(json.dumps(r), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["c2", "c1", "c3", "c3z", "c4", "c5"], default="c2")
    ap.add_argument("--c4-count", type=int, default=4096)
    ap.add_argument("--rates", type=float, nargs="+", default=[10, 30, 100, 300])
    ap.add_argument("--serve-seconds", type=float, default=10.0)
    ap.add_argument("--slots", type=int, default=32,
                    help="requests the server keeps admitted at once (c5)")
    ap.add_argument("--no-extras", action="store_true",
                    help="default line: skip the c4 batch, c5 serving and c3 accuracy summaries")
    ap.add_argument("--extra-rates", type=float, nargs="+", default=[10, 30, 100])
    ap.add_argument("--extra-serve-seconds", type=float, default=6.0)
    ap.add_argument("--c3-width", type=int, default=32768,
                    help="diagonals of the c3/c3z accuracy sample in the default line")
    ap.add_argument("--reanchor-k", type=int, default=1024)
    ap.add_argument("--fp64-steps", type=int, default=3)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference_arm(args, world)
        return
    if args.workload in ("c4", "c5") and int(os.environ.get("RANK", "0")) != 0:
        return  # replicas: rank 0 drives every GPU; the other ranks have no work
    if args.workload == "c4":
        run_batch_workload(args)
        return
    if args.workload == "c5":
        run_serving_workload(args)
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, world)
    finally:
        if world > 1:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
