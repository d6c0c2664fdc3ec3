"""The FP32 join's tile space on CPU: fp32_tile_plan (host) and fp32_tile_of
(the kernel's tile -> (band, column segment) map, also host-callable) must
cover every cell (diagonal g in [g_lo, g_hi), column j < PL - g) exactly once,
in band pairs (k, nbands-1-k), for full joins, diagonal partitions and tiny
profiles.  Compiled with nvcc as a host program against libmpgpu.so."""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

import thesiscode_b200 as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "thesiscode_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "mp_kernels.h"
using namespace mpgpu;

// returns 0 when the tiles of (PL, g_lo, g_hi, K) cover the triangle exactly once
static int check(int64_t PL, int64_t g_lo, int64_t g_hi, int64_t K) {
    const int R = 8;
    const int64_t span = 32 * R;
    Fp32TileParams P{};
    P.PL = PL; P.g_lo = g_lo; P.g_hi = g_hi; P.K = K;
    int64_t ntiles = 0;
    fp32_tile_plan(PL, g_lo, g_hi, K, R, P.nbands, P.seg_per_pair, ntiles);
    const int64_t ndiag = g_hi > g_lo ? g_hi - g_lo : 0;
    if (P.nbands != (ndiag + span - 1) / span) return 1;
    std::vector<unsigned char> hits((size_t)(PL + 1) * (size_t)(PL + 1), 0);
    std::vector<int> band_seen((size_t)P.nbands + 1, 0);
    for (int64_t lt = 0; lt < ntiles; ++lt) {
        int64_t band = -1, seg = -1;
        if (!fp32_tile_of(P, lt, span, band, seg)) continue;
        if (band < 0 || band >= P.nbands || seg < 0) return 2;
        // the pair of tile lt holds bands p and nbands - 1 - p
        const int64_t p = lt / P.seg_per_pair;
        if (band != p && band != P.nbands - 1 - p) return 3;
        band_seen[band] = 1;
        const int64_t gb = g_lo + band * span, jmax = PL - gb;
        const int64_t j0 = seg * K, j1 = j0 + K < jmax ? j0 + K : jmax;
        for (int64_t d = 0; d < span; ++d) {
            const int64_t g = gb + d;
            if (g >= g_hi) break;
            for (int64_t j = j0; j < j1 && j < PL - g; ++j)
                if (++hits[(size_t)g * (size_t)(PL + 1) + (size_t)j] > 1) return 4;
        }
    }
    for (int64_t b = 0; b < P.nbands; ++b)
        if (!band_seen[b] && PL - (g_lo + b * span) > 0) return 5;
    for (int64_t g = g_lo; g < g_hi; ++g)
        for (int64_t j = 0; j < PL - g; ++j)
            if (hits[(size_t)g * (size_t)(PL + 1) + (size_t)j] != 1) return 6;
    return 0;
}

int main() {
    int bad = 0, cases = 0;
    const int64_t Ks[] = {8, 64, 256, 1024, 4096};
    const int64_t PLs[] = {1, 2, 17, 255, 256, 257, 511, 1000, 2049, 2600};
    for (int64_t PL : PLs)
        for (int64_t K : Ks) {
            const int64_t excl = 16;
            // full join, a diagonal partition pair's ranges, a single diagonal
            const int64_t ranges[][2] = {{excl + 1, PL}, {excl + 1, excl + 1 + PL / 3},
                                         {PL / 2, PL}, {PL / 3, PL / 3 + 1}, {0, PL}};
            for (auto& r : ranges) {
                const int64_t lo = r[0], hi = r[1] < PL ? r[1] : PL;
                ++cases;
                const int rc = check(PL, lo, hi, K);
                if (rc) {
                    std::printf("FAIL PL=%lld lo=%lld hi=%lld K=%lld code=%d\n", (long long)PL,
                                (long long)lo, (long long)hi, (long long)K, rc);
                    ++bad;
                }
            }
        }
    std::printf("%d cases, %d failed\n", cases, bad);
    return bad ? 1 : 0;
}
"""


def test_tiles_cover_each_cell_exactly_once(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    mp.load_library()  # built library present
    src = tmp_path / "tiles.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "tiles"
    libdir = os.path.dirname(mp.LIB_PATH)
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets", f"-I{CSRC}", str(src), "-o", str(exe),
                    f"-L{libdir}", "-lmpgpu", "-Xlinker", f"-rpath={libdir}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failed" in r.stdout
