"""The guarded form's neighbour pick on CPU (fp32_pick_neighbour in
thesiscode_b200/csrc/mp_kernels.h, the code its finalisation runs, compiled
with nvcc as a host program): of the candidates q in [lo, lo + n) that are
partners of window i in the join (0 <= q < PL and g_lo <= |i - q| < g_hi), it
returns the one whose window has the largest centred correlation with window
i, never a flat (NaN) one, and -1 when none qualifies.  Checked against a
direct long-double computation over random windows, candidate ranges that
reach past either end of the profile and past the diagonal range, and a
series with constant stretches."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "thesiscode_b200", "csrc")

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>
#include "mp_kernels.h"
using namespace mpgpu;

int main() {
    std::mt19937_64 rng(11);
    std::normal_distribution<double> N(0.0, 1.0);
    int bad = 0, cases = 0, none = 0;
    for (int64_t m : {4, 8, 17, 64, 100}) {
        for (int64_t n : {40, 300, 2000}) {
            if (n < 2 * m) continue;
            // a random walk with constant stretches, padded past its end
            std::vector<double> A(n + kPickSlots, 0.0);
            double v = 0.0;
            for (int64_t t = 0; t < n; ++t) {
                if (!((t / 97) % 5 == 3)) v += N(rng);
                A[t] = v;
            }
            const int64_t PL = n - m + 1;
            std::vector<double> mean(PL), norm(PL);
            for (int64_t w = 0; w < PL; ++w) {
                long double s = 0, ss = 0;
                for (int64_t t = 0; t < m; ++t) s += A[w + t];
                mean[w] = (double)(s / m);
                for (int64_t t = 0; t < m; ++t) ss += (A[w + t] - mean[w]) * (A[w + t] - mean[w]);
                norm[w] = ss > 0 ? (double)(1.0L / std::sqrt(ss)) : NAN;
            }
            auto corr = [&](int64_t i, int64_t q) {
                long double c = 0;
                for (int64_t t = 0; t < m; ++t)
                    c += (long double)(A[i + t] - mean[i]) * (A[q + t] - mean[q]);
                return c * norm[q];
            };
            for (int trial = 0; trial < 400; ++trial) {
                ++cases;
                const int64_t i = (int64_t)(rng() % PL);
                const int cnt = 1 + (int)(rng() % kPickSlots);
                const int64_t lo = (int64_t)(rng() % (PL + 2 * kPickSlots)) - kPickSlots;
                const int64_t g_lo = (int64_t)(rng() % (m / 4 + 2));
                const int64_t g_hi = g_lo + 1 + (int64_t)(rng() % PL);
                int64_t want = -1;
                long double best = 0;
                for (int64_t q = lo; q < lo + cnt; ++q) {
                    const int64_t g = q > i ? q - i : i - q;
                    if (q < 0 || q >= PL || g < g_lo || g >= g_hi || std::isnan(norm[q])) continue;
                    const long double c = corr(i, q);
                    if (want < 0 || c > best) { best = c; want = q; }
                }
                const int64_t got =
                    fp32_pick_neighbour(A.data(), mean.data(), norm.data(), m, PL, g_lo, g_hi, i, lo, cnt);
                bool ok;
                if (want < 0) {
                    ok = got == -1;
                    ++none;
                } else {
                    const int64_t g = got > i ? got - i : i - got;
                    ok = got >= lo && got < lo + cnt && got >= 0 && got < PL && g >= g_lo && g < g_hi &&
                         !std::isnan(norm[got]) &&
                         corr(i, got) >= best - 1e-9L * (1 + std::fabs((double)best));
                }
                if (!ok && bad++ < 5)
                    std::printf("m=%lld n=%lld i=%lld lo=%lld cnt=%d g=[%lld,%lld) got %lld want %lld\n",
                                (long long)m, (long long)n, (long long)i, (long long)lo, cnt,
                                (long long)g_lo, (long long)g_hi, (long long)got, (long long)want);
            }
        }
    }
    std::printf("%d cases (%d without a candidate), %d failed\n", cases, none, bad);
    return bad ? 1 : 0;
}
"""


def test_pick_equals_direct_best_candidate(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "pick.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "pick"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    f"-I{CSRC}", str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 failed" in r.stdout
