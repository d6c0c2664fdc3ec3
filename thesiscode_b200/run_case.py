"""Runs one self-join of a seeded random walk through the C ABI and prints its
kernel phase times -- a fixed, small command for profilers and quick checks.

    python -m thesiscode_b200.run_case --n 262144 --m 256 --precision fp32 [--k 1024]
    python -m thesiscode_b200.run_case --n 262144 --m 256 --prescrimp 0.25
"""
from __future__ import annotations

import argparse
import time

import numpy as np

import thesiscode_b200 as mp
from thesiscode_b200 import workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262_144)
    ap.add_argument("--m", type=int, default=256)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--precision", choices=["fp32", "fp64", "guarded"], default="fp32")
    ap.add_argument("--k", type=int, default=1024, help="FP32 re-anchor interval")
    ap.add_argument("--prescrimp", type=float, default=None, metavar="STRIDE",
                    help="run PreSCRIMP with this stride instead of the self-join")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args()
    x = workloads.random_walk(a.n, a.seed)
    prec = {"fp32": mp.FP32_REANCHOR, "fp64": mp.FP64, "guarded": mp.FP32_GUARDED}[a.precision]
    with mp.Context(0) as ctx:
        ctx.set_phase_timing(True)
        if a.prescrimp is not None:
            for _ in range(a.repeat):
                t0 = time.perf_counter()
                p = ctx.prescrimp(x, a.m, a.prescrimp)
                ms = (time.perf_counter() - t0) * 1e3
                print(f"prescrimp n={a.n} m={a.m} stride={a.prescrimp}: {ms:.3f} ms, "
                      f"min distance {float(np.sqrt(np.nanmin(p.dist2))):.6f}")
            return
        for _ in range(a.repeat):
            p = ctx.selfjoin(x, a.m, precision=prec, reanchor_k=a.k)
            prep, join, fin = ctx.last_phase_ms()
            cells = mp.cells(a.n, a.m)
            print(f"{a.precision} n={a.n} m={a.m}: prep {prep:.3f} ms, join {join:.3f} ms "
                  f"({cells / (join * 1e-3):.3e} cells/s), finalize {fin:.3f} ms, "
                  f"min distance {float(np.sqrt(p.dist2.min())):.6f}")


if __name__ == "__main__":
    main()
