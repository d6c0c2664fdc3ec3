"""Profile error of the FP32 re-anchored form against the FP64 form, per
workload and re-anchor interval K.

The FP64 form returns the reference's own values (ScrimpVertBlocked with its
IEEE arithmetic, scrimppp/src/ScrimpVertBlocked.cpp:89-195); the error of a
window is the relative error of its distance, |sqrt(d2_32) - sqrt(d2_64)| /
sqrt(d2_64).

The reference's FP64 values are not always accurate themselves: its window
variance is a difference of prefix sums (scrimppp/src/ScrimpSequOpt.cpp:58-72)
that grow with the series, so for nearly flat windows of a long series (a few
walk samples and a constant stretch) the variance -- and every score of the
window -- carries large rounding error, and windows wholly inside a constant
stretch at a non-zero level get a variance of rounding noise (~1e-11) instead
of 0.  Every window whose two results differ by more than 1e-4 is therefore
judged against the distances of the chosen pairs computed directly (centred
two-pass FP64 dot products, independent of both forms): the window is
"reference-inaccurate" when the FP64 value is more than 1e-6 away from the
direct distance of its own pair, when that pair is flat, when the FP64 form
found no neighbour although the FP32 form's pair is a valid one, or when the
FP32 form's pair is closer than the FP64 form's (the reference's rounding hid
the nearest neighbour).  Windows
wholly inside a constant stretch ("pseudo-flat") are counted apart: the FP32
form detects them as flat and gives them the flat result (d2 = 2m + 2, index
0) that the reference gives exactly flat windows.

    python -m thesiscode_b200.error_report --workloads c1 c2 c3 c3z --ks 64 256 1024
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

import thesiscode_b200 as mp
from thesiscode_b200 import workloads as wl


def load(name: str):
    """(x, m, constant segments [(start, length)], description) of a workload."""
    if name == "c1":
        x, m = wl.c1()
        return x, m, [], "c1: random walk n=65,536 seed 0, m=400"
    if name == "c2":
        x, m = wl.c2()
        return x, m, [], "c2: random walk n=1,048,576 seed 1, m=256"
    if name in ("c3", "c3z"):
        zero = name == "c3z"
        x, m, info = wl.c3(zero_level=zero)
        segs = [(s, L) for kind, s, L in info if kind == "flat"]
        lvl = "zero-level" if zero else "non-zero-level"
        return x, m, segs, (f"{name}: random walk n=8,388,608 seed 2, m=1024, 32 planted sine "
                            f"motifs, 16 {lvl} constant segments of 2m")
    raise ValueError(name)


def inside_constant(PL: int, m: int, segs) -> np.ndarray:
    """Windows lying wholly inside one of the constant segments."""
    mask = np.zeros(PL, dtype=bool)
    for s, L in segs:
        lo, hi = s, min(s + L - m + 1, PL)
        if hi > lo:
            mask[lo:hi] = True
    return mask


def pair_distance(x, m: int, i: int, j: int) -> float:
    """z-normalised distance of windows i and j from centred two-pass FP64 dot
    products (NaN when either window is flat)."""
    a = x[i:i + m] - np.mean(x[i:i + m])
    b = x[j:j + m] - np.mean(x[j:j + m])
    va, vb = float(a @ a), float(b @ b)
    if va == 0.0 or vb == 0.0:
        return float("nan")
    rho = float(a @ b) / np.sqrt(va * vb)
    return float(np.sqrt(max(2.0 * m * (1.0 - rho), 0.0)))


def stretch_zone(PL: int, m: int, segs, K: int) -> np.ndarray:
    """Windows that overlap a constant stretch or start within K windows
    after one: the cells of their diagonals may follow, within one re-anchor
    interval, cells of windows that straddle the stretch's edges, whose
    centred dot products are orders of magnitude larger."""
    zone = np.zeros(PL, dtype=bool)
    for s, L in segs:
        zone[max(s - m - K, 0):min(s + L + K, PL)] = True
    return zone


def compare(x, m, segs, p64, p32, zero_level: bool, tol: float = 1e-4, K: int = 1024):
    PL = x.size - m + 1
    none = np.sqrt(2.0 * m + 2.0)  # distance of a window without neighbour
    d64 = np.sqrt(np.abs(p64.dist2))
    d32 = np.sqrt(np.abs(p32.dist2))
    const = inside_constant(PL, m, segs)
    pseudo = const if not zero_level else np.zeros(PL, dtype=bool)
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.abs(d32 - d64) / d64
    rel[pseudo] = 0.0
    over = np.nonzero(rel > tol)[0]
    ref_bad = np.zeros(PL, dtype=bool)
    worst_vs_direct = 0.0
    worse_neighbour = 0
    examples = []
    for i in over:
        e64 = pair_distance(x, m, i, int(p64.index[i])) if d64[i] < none else None
        e32 = pair_distance(x, m, i, int(p32.index[i])) if d32[i] < none else None
        if e64 is not None and (not np.isfinite(e64) or abs(d64[i] - e64) > 1e-6 * e64):
            ref_bad[i] = True
        if e64 is None and e32 is not None and np.isfinite(e32) and e32 < none * (1 - 1e-6):
            ref_bad[i] = True
        if (e64 is not None and e32 is not None and np.isfinite(e64) and np.isfinite(e32)
                and e32 < e64 * (1 - 1e-6)):
            ref_bad[i] = True  # the other form found a closer neighbour than the reference
        if e32 is not None and np.isfinite(e32) and e32 > 0:
            worst_vs_direct = max(worst_vs_direct, abs(d32[i] - e32) / e32)
            if e64 is not None and np.isfinite(e64) and e32 > e64 * (1 + tol):
                worse_neighbour += 1
                if len(examples) < 5:
                    examples.append({"window": int(i), "fp64_index": int(p64.index[i]),
                                     "fp32_index": int(p32.index[i]), "fp64": float(d64[i]),
                                     "fp32": float(d32[i]), "direct_fp64_pair": e64,
                                     "direct_fp32_pair": e32})
    ok = ~(pseudo | ref_bad)
    rel_ok = rel[ok]
    zone = stretch_zone(PL, m, segs, K)
    near = zone | zone[p64.index.clip(0, PL - 1)] | zone[p32.index.clip(0, PL - 1)]
    far_ok = ok & ~near
    rep = {
        "windows": PL,
        "max_rel_all": float(np.max(rel[~pseudo])),
        "max_rel": float(np.max(rel_ok)) if rel_ok.size else 0.0,
        "mean_rel": float(np.mean(rel_ok)) if rel_ok.size else 0.0,
        "p99_rel": float(np.percentile(rel_ok, 99)) if rel_ok.size else 0.0,
        "index_agreement": float(np.mean(p32.index[ok] == p64.index[ok])) if ok.any() else 1.0,
        "windows_over_tol": int(over.size),
        "reference_inaccurate": int(ref_bad.sum()),
        "fp32_max_rel_vs_direct_on_those": worst_vs_direct,
        "fp32_neighbour_worse_than_fp64": worse_neighbour,
        "near_stretch_windows": int(near.sum()),
        "max_rel_far_from_stretches": float(np.max(rel[far_ok])) if far_ok.any() else 0.0,
        "max_rel_near_stretches": float(np.max(rel[ok & near])) if (ok & near).any() else 0.0,
    }
    if examples:
        rep["worse_neighbour_examples"] = examples
    if zero_level and const.any():
        flat_d2 = 2.0 * m + 2.0
        rep["flat_windows"] = int(const.sum())
        rep["flat_convention_fp64"] = bool(np.all(p64.dist2[const] == flat_d2)
                                           and np.all(p64.index[const] == 0))
        rep["flat_convention_fp32"] = bool(np.all(p32.dist2[const] == flat_d2)
                                           and np.all(p32.index[const] == 0))
        found = p32.dist2[~const] < flat_d2
        rep["no_window_points_at_flat_fp32"] = bool(not np.any(const[p32.index[~const][found]]))
    if not zero_level and const.any():
        rep["pseudo_flat_windows"] = int(const.sum())
        rep["pseudo_flat_fp32_is_flat_result"] = bool(np.all(p32.dist2[const] == 2.0 * m + 2.0))
    return rep


def run(names, ks, device: int = 0, out=sys.stdout, forms=("fp32",)):
    with mp.Context(device) as ctx:
        ctx.set_phase_timing(True)
        for name in names:
            x, m, segs, desc = load(name)
            cells = mp.cells(x.size, m)
            t0 = time.perf_counter()
            p64 = ctx.selfjoin(x, m, precision=mp.FP64)
            wall64 = time.perf_counter() - t0
            join64 = ctx.last_phase_ms()[1]
            for form, k in [(f, k) for f in forms for k in ks]:
                prec = mp.FP32_GUARDED if form == "guarded" else mp.FP32_REANCHOR
                p32 = ctx.selfjoin(x, m, precision=prec, reanchor_k=k)
                join32 = ctx.last_phase_ms()[1]
                rep = {"workload": name, "form": form, "description": desc, "m": m, "reanchor_k": k,
                       "cells": cells,
                       "fp64_join_ms": join64, "fp64_wall_s": wall64,
                       "fp32_join_ms": join32,
                       "fp64_cells_per_s": cells / (join64 * 1e-3),
                       "fp32_cells_per_s": cells / (join32 * 1e-3)}
                if form == "guarded":
                    rep["near_duplicates_recomputed"] = ctx.last_near_duplicates
                rep.update(compare(x, m, segs, p64, p32, name == "c3z", K=k))
                print(json.dumps(rep), file=out, flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--workloads", nargs="+", default=["c1", "c2", "c3", "c3z"])
    ap.add_argument("--ks", nargs="+", type=int, default=[64, 256, 1024])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None, help="append JSON lines here too")
    ap.add_argument("--forms", nargs="+", default=["fp32"], choices=["fp32", "guarded"],
                    help="fp32: the re-anchored form; guarded: with FP64 tiles around "
                         "ill-conditioned windows")
    a = ap.parse_args(argv)
    if a.out:
        with open(a.out, "a") as f:
            class Tee:
                def write(self, s):
                    sys.stdout.write(s)
                    f.write(s)

                def flush(self):
                    sys.stdout.flush()
                    f.flush()
            run(a.workloads, a.ks, a.device, Tee(), tuple(a.forms))
    else:
        run(a.workloads, a.ks, a.device, forms=tuple(a.forms))


if __name__ == "__main__":
    main()
