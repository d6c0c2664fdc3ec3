"""Runs one self-join of a seeded random walk through the C ABI and prints its
kernel phase times -- a fixed, small command for profilers and quick checks.

    python -m thesiscode_b200.run_case --n 262144 --m 256 --precision fp32 [--k 1024]
"""
from __future__ import annotations

import argparse

import numpy as np

import thesiscode_b200 as mp
from thesiscode_b200 import workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=262_144)
    ap.add_argument("--m", type=int, default=256)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--k", type=int, default=1024, help="FP32 re-anchor interval")
    ap.add_argument("--repeat", type=int, default=1)
    a = ap.parse_args()
    x = workloads.random_walk(a.n, a.seed)
    prec = mp.FP32_REANCHOR if a.precision == "fp32" else mp.FP64
    with mp.Context(0) as ctx:
        ctx.set_phase_timing(True)
        for _ in range(a.repeat):
            p = ctx.selfjoin(x, a.m, precision=prec, reanchor_k=a.k)
            prep, join, fin = ctx.last_phase_ms()
            cells = mp.cells(a.n, a.m)
            print(f"{a.precision} n={a.n} m={a.m}: prep {prep:.3f} ms, join {join:.3f} ms "
                  f"({cells / (join * 1e-3):.3e} cells/s), finalize {fin:.3f} ms, "
                  f"min distance {float(np.sqrt(p.dist2.min())):.6f}")


if __name__ == "__main__":
    main()
