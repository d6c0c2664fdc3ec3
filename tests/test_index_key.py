"""The FP64 form's index key (idx_key_f64, thesiscode_b200/csrc/mp_common.cuh)
on CPU.  Profiles are max-merged on this 64-bit key, so it must order
candidates by v = m - score (half the squared distance; smaller v wins), break
equal high parts toward the smaller neighbour, put v <= 0 above every v > 0
(and order v <= 0 by |v| up to inf, for the huge scores of near-constant
windows),
keep ~33 mantissa bits at idx_bits = 24 (ties only within ~1.2e-10 relative),
and give back the neighbour from its low bits.  Compiled with nvcc as a host
program (the key function is host-callable)."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "thesiscode_b200", "csrc")

PROGRAM = r"""
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <random>
#include "mp_common.cuh"
using namespace mpgpu;

static int fails = 0;
#define CHECK(c, ...) do { if (!(c)) { if (fails++ < 10) { std::printf(__VA_ARGS__); std::printf("\n"); } } } while (0)

static uint64_t nb_of(unsigned long long key, int idx_bits) {
    const unsigned long long lowmask = (1ull << idx_bits) - 1ull;
    return lowmask - (key & lowmask);
}

int main() {
    std::mt19937_64 rng(12345);
    for (int64_t m : {8LL, 64LL, 256LL, 400LL, 1024LL, 4096LL}) {
        const long long vlo = key_vlo_bits(m);
        // vlo = 2^(t-64) with 2^t > 2m + 2 >= 2^(t-1)
        const int t = (int)((vlo >> 52) - 1023 + 64);
        CHECK(std::ldexp(1.0, t) > 2.0 * m + 2.0 && std::ldexp(1.0, t - 1) <= 2.0 * m + 2.0,
              "vlo m=%lld t=%d", (long long)m, t);
        for (int idx_bits : {bits_for(1000), bits_for(1 << 20), bits_for((1 << 24) - 1)}) {
            const uint64_t maxnb = (1ull << idx_bits) - 1;
            std::uniform_real_distribution<double> U(-1.0, 1.0);
            for (int it = 0; it < 20000; ++it) {
                // two candidates' scores in [-m, m] (correlation in [-1, 1])
                const double s1 = m * U(rng), s2 = m * U(rng);
                const uint64_t n1 = rng() & maxnb, n2 = rng() & maxnb;
                const unsigned long long k1 = idx_key_f64(s1, (double)m, n1, idx_bits, vlo);
                const unsigned long long k2 = idx_key_f64(s2, (double)m, n2, idx_bits, vlo);
                CHECK(nb_of(k1, idx_bits) == n1, "decode m=%lld", (long long)m);
                const double v1 = m - s1, v2 = m - s2;
                // clearly smaller v (beyond 2^-30 relative) -> larger key
                if (v1 > 0 && v2 > 0 && v1 < v2 * (1.0 - std::ldexp(1.0, -30)))
                    CHECK(k1 > k2, "order v1=%.17g v2=%.17g", v1, v2);
                if (v1 <= 0 && v2 > 0) CHECK(k1 > k2, "region v1=%.17g v2=%.17g", v1, v2);
            }
            // equal scores: the smaller neighbour has the larger key
            for (int it = 0; it < 2000; ++it) {
                const double s = m * U(rng);
                const uint64_t a = rng() & maxnb, b = rng() & maxnb;
                if (a == b) continue;
                const unsigned long long ka = idx_key_f64(s, (double)m, a, idx_bits, vlo);
                const unsigned long long kb = idx_key_f64(s, (double)m, b, idx_bits, vlo);
                CHECK((a < b) == (ka > kb), "tie s=%.17g a=%llu b=%llu", s,
                      (unsigned long long)a, (unsigned long long)b);
            }
            // Resolution of the high part: 64 - idx_bits - 1 (region) - 6 (exponent)
            // mantissa bits (33 at idx_bits = 24), i.e. |v|'s bit pattern in quanta
            // of 2^(52 - mantissa bits).  Two v one quantum apart never share a high
            // part.  The key sees v = m - score; score = -v with m = 0 keeps v exact.
            const int mant = 64 - idx_bits - 1 - 6;
            if (idx_bits == 24) CHECK(mant == 33, "mantissa bits %d", mant);
            const long long quantum = 1ll << (52 - mant);
            for (int it = 0; it < 20000; ++it) {
                const double v = std::ldexp(1.0 + U(rng) * 0.5, -(int)(rng() % 30)) * m;
                const long long b2 = f64_bits(v) + quantum;
                double v2;
                std::memcpy(&v2, &b2, sizeof v2);
                const unsigned long long ka = idx_key_f64(-v, 0.0, 0, idx_bits, vlo);
                const unsigned long long kb = idx_key_f64(-v2, 0.0, 0, idx_bits, vlo);
                CHECK((ka >> idx_bits) > (kb >> idx_bits), "resolution v=%.17g", v);
            }
            // monotone across binade boundaries of v
            for (int e = -40; e < t; ++e) {
                const double below = std::nextafter(std::ldexp(1.0, e), 0.0);
                const double at = std::ldexp(1.0, e);
                if (at >= 2.0 * m + 2.0) break;
                const unsigned long long kb_ = idx_key_f64(m - below, (double)m, 0, idx_bits, vlo);
                const unsigned long long ka_ = idx_key_f64(m - at, (double)m, 0, idx_bits, vlo);
                if (m - (m - below) < m - (m - at)) CHECK(kb_ >= ka_, "binade e=%d", e);
            }
            // v <= 0 (score >= m, e.g. the huge scores of a window whose variance
            // rounds to a tiny positive value): the key grows with |v| over the
            // whole double range -- through the end of the fine region at
            // 2^(t-32) and up to inf -- strictly once |v| > vlo, and stays above
            // every v > 0.  score = |v| with m = 0 keeps v exact.
            {
                const unsigned long long top_pos =
                    idx_key_f64(-std::ldexp(1.0, t - 64), 0.0, 0, idx_bits, vlo) >> idx_bits;
                unsigned long long prev = idx_key_f64(0.0, 0.0, 0, idx_bits, vlo) >> idx_bits;
                CHECK(prev > top_pos, "region at v = 0");
                for (int e = t - 70; e < 1023; ++e) {
                    for (double f : {1.0, 1.3, 1.7}) {
                        const double a = std::ldexp(f, e);
                        const unsigned long long k = idx_key_f64(a, 0.0, 0, idx_bits, vlo) >> idx_bits;
                        if (a > std::ldexp(1.0, t - 64)) CHECK(k > prev, "neg order |v|=%.17g", a);
                        else CHECK(k == prev, "neg clamp |v|=%.17g", a);
                        prev = k;
                    }
                }
                const double edge = std::ldexp(1.0, t - 32);
                const unsigned long long kin =
                    idx_key_f64(std::nextafter(edge, 0.0), 0.0, 0, idx_bits, vlo) >> idx_bits;
                const unsigned long long kout = idx_key_f64(edge, 0.0, 0, idx_bits, vlo) >> idx_bits;
                CHECK(kout > kin, "fine/coarse edge");
                const unsigned long long kinf =
                    idx_key_f64(HUGE_VAL, 0.0, 0, idx_bits, vlo) >> idx_bits;
                const unsigned long long kmax = idx_key_f64(DBL_MAX, 0.0, 0, idx_bits, vlo) >> idx_bits;
                CHECK(kinf >= kmax && kmax >= prev, "top of the range");
                CHECK(kinf < (1ull << (64 - idx_bits)), "field overflow");
            }
        }
    }
    std::printf("%d failed\n", fails);
    return fails ? 1 : 0;
}
"""


def test_index_key_orders_and_decodes(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "key.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "key"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    f"-I{CSRC}", str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failed" in r.stdout


THRESHOLD_PROGRAM = r"""
#include <cstdio>
#include <random>
#include "mp_common.cuh"
#include "mp_kernels.h"
using namespace mpgpu;

static int fails = 0;
#define CHECK(c, ...) do { if (!(c)) { if (fails++ < 10) { std::printf(__VA_ARGS__); std::printf("\n"); } } } while (0)

int main() {
    std::mt19937_64 rng(777);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    long long checked = 0;
    for (int64_t m : {4LL, 64LL, 256LL, 1024LL, 8192LL}) {
        const long long vlo = key_vlo_bits(m);
        for (int idx_bits : {bits_for(100), bits_for(1 << 20), bits_for((1 << 24) - 1),
                             bits_for((1ull << 31) - 1)}) {
            const double eps = fp64_threshold_eps(idx_bits), tiny = fp64_threshold_tiny((double)m);
            const int mant = 57 - idx_bits;
            for (int it = 0; it < 200000; ++it) {
                // a merged score c (correlation in (-1/m, 1], some near 1) and a
                // candidate x whose v lies within a few key quanta of c's
                const int e = -(int)(rng() % 45);
                double vc = std::ldexp(0.5 + U(rng), e) * (double)m;
                if (rng() % 16 == 0) vc = -vc * 1e-3;  // score above m (rounding)
                const double sc = (double)m - vc;
                const double q = std::ldexp(std::fabs(vc), -mant);
                const double vx = vc + (U(rng) * 6.0 - 3.0) * q;
                const double sx = (double)m - vx;
                const unsigned long long kc = idx_key_f64(sc, (double)m, 0, idx_bits, vlo) >> idx_bits;
                const unsigned long long kx = idx_key_f64(sx, (double)m, 0, idx_bits, vlo) >> idx_bits;
                const double t = fp64_threshold_below(sc, (double)m, eps, tiny);
                CHECK(t < sc, "threshold not below the score: m=%lld s=%.17g t=%.17g",
                      (long long)m, sc, t);
                if (kx >= kc) {
                    ++checked;
                    CHECK(sx > t, "pruned a tying key: m=%lld bits=%d sc=%.17g sx=%.17g t=%.17g",
                          (long long)m, idx_bits, sc, sx, t);
                }
            }
        }
    }
    std::printf("%lld tying candidates, %d failed\n", checked, fails);
    return fails ? 1 : 0;
}
"""


def test_fp64_threshold_keeps_every_tying_key(tmp_path):
    """The FP64 join skips the selection of a cell whose score does not exceed
    its entry's threshold.  Thresholds sit below a merged score by more than the
    index key resolves, so a candidate whose key could still tie or beat that
    score's key always exceeds them: skipping cannot change either key."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "thr.cu"
    src.write_text(THRESHOLD_PROGRAM)
    exe = tmp_path / "thr"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    f"-I{CSRC}", str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 failed" in r.stdout
