"""The guarded form's hazard rule on CPU (hazard_block_minima / hazard_flag in
thesiscode_b200/csrc/mp_kernels.h, the code the hazard kernels run, compiled
with nvcc as a host program): window w is a hazard exactly when it is flat
(NaN inverse norm) or its inverse norm exceeds 16 times the smallest finite
inverse norm among windows [w - (blk - 1), w].  Checked against a direct
minimum over that range, with flat windows, single-window blocks, ragged last
blocks and blocks longer than the profile."""
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
    std::mt19937_64 rng(7);
    int bad = 0, cases = 0;
    for (int64_t PL : {1, 2, 5, 64, 257, 1000, 4099}) {
        for (int64_t blk : {1, 2, 3, 17, 64, 256, 5000}) {
            for (int trial = 0; trial < 3; ++trial) {
                ++cases;
                std::vector<double> nn(PL), pre(PL), suf(PL);
                std::lognormal_distribution<double> L(0.0, 1.2);
                for (auto& v : nn) {
                    const unsigned r = rng() % 100;
                    v = r < 5 ? NAN : (r < 8 ? 40.0 * L(rng) : L(rng));  // flats, spikes
                }
                const int64_t nb = (PL + blk - 1) / blk;
                for (int64_t b = 0; b < nb + 1; ++b)  // one block past the end does nothing
                    hazard_block_minima(nn.data(), PL, blk, b, pre.data(), suf.data());
                for (int64_t w = 0; w < PL; ++w) {
                    double mn = NAN;
                    const int64_t lo = w - (blk - 1) > 0 ? w - (blk - 1) : 0;
                    for (int64_t i = lo; i <= w; ++i) mn = std::fmin(mn, nn[i]);
                    const int want = (std::isnan(nn[w]) || nn[w] > 16.0 * mn) ? 1 : 0;
                    const int got = hazard_flag(nn.data(), pre.data(), suf.data(), blk, w);
                    if (got != want) {
                        if (bad++ < 5)
                            std::printf("PL=%lld blk=%lld w=%lld got %d want %d\n", (long long)PL,
                                        (long long)blk, (long long)w, got, want);
                    }
                }
            }
        }
    }
    std::printf("%d cases, %d failed\n", cases, bad);
    return bad ? 1 : 0;
}
"""


def test_hazard_flags_equal_a_direct_sliding_minimum(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "hazard.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "hazard"
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    f"-I{CSRC}", str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 failed" in r.stdout
