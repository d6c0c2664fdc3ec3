"""Seeded synthetic series for the five workloads of this path.

All inputs are generated (no dataset exists for them): random walks
x = cumsum(N(0, 1)) drawn with numpy's default_rng(seed).

  c1  n = 65,536, seed 0, m = 400                 (the reference's CPU case)
  c2  n = 1,048,576, seed 1, m = 256              (the single-GPU headline)
  c3  n = 8,388,608, seed 2, m = 1024, with 32 planted motifs
      (3*sin(2*pi*t/P + phi) + N(0, 0.1) over m samples, P = m/4) and
      16 constant segments of length 2m (drift and flat-window stress)
  c4  4,096 FP32-input walks, lengths log-uniform in [2048, 262144],
      m uniform in {64, 128, 256}, seed 3           (batched joins)
  c5  Poisson request stream, lengths log-uniform in [1024, 1048576],
      m uniform in {32, 64, 128, 256, 512, 1024}, seed 4   (serving)
"""
from __future__ import annotations

import numpy as np


def random_walk(n: int, seed: int) -> np.ndarray:
    return np.cumsum(np.random.default_rng(seed).standard_normal(n))


def c1():
    return random_walk(65_536, 0), 400


def c2():
    return random_walk(1_048_576, 1), 256


def c3(n: int = 8_388_608, m: int = 1024, zero_level: bool = False, seed: int = 2):
    """Random walk with 32 planted sine motifs and 16 constant segments.

    The constant segments hold the walk's value at their start (non-zero level)
    or 0.0 with ``zero_level``.  Returns (x, m, info)."""
    rng = np.random.default_rng(seed)
    x = np.cumsum(rng.standard_normal(n))
    nmotif, nflat = 32, 16
    lens = [m] * nmotif + [2 * m] * nflat
    kinds = ["motif"] * nmotif + ["flat"] * nflat
    order = rng.permutation(len(lens))
    slot = n // len(lens)
    info = []
    for k, which in enumerate(order):
        L = lens[which]
        start = k * slot + int(rng.integers(0, max(slot - L, 1)))
        if kinds[which] == "motif":
            P = m / 4.0
            phi = rng.uniform(0.0, 2.0 * np.pi)
            t = np.arange(L)
            x[start:start + L] += 3.0 * np.sin(2 * np.pi * t / P + phi) + rng.normal(0, 0.1, L)
        else:
            x[start:start + L] = 0.0 if zero_level else x[start]
        info.append((kinds[which], start, L))
    return x, m, info


def c4(count: int = 4096, seed: int = 3):
    """List of (float32 series, m)."""
    rng = np.random.default_rng(seed)
    lens = np.floor(np.exp(rng.uniform(np.log(2048), np.log(262_144), count))).astype(np.int64)
    ms = rng.choice([64, 128, 256], size=count)
    out = []
    for i in range(count):
        s = np.cumsum(rng.standard_normal(int(lens[i]))).astype(np.float32)
        out.append((s, int(ms[i])))
    return out


def c5_stream(rate_hz: float, duration_s: float, seed: int = 4):
    """Poisson arrivals: list of (arrival_time_s, n, m, series_seed)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate_hz)
        if t >= duration_s:
            break
        n = int(np.floor(np.exp(rng.uniform(np.log(1024), np.log(1_048_576)))))
        m = int(rng.choice([32, 64, 128, 256, 512, 1024]))
        if n < 2 * m:
            n = 2 * m
        out.append((t, n, m, int(rng.integers(0, 2**31 - 1))))
    return out
