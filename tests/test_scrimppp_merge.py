"""SCRIMP++'s final profile on CPU: the merge rule of the gpu_scrimppp variant
(thesiscode_b200/csrc/host/scrimppp_merge.hpp, compiled with g++) applied to
the PreSCRIMP restatement and the oracle's exact join must give the reference's
own final scrimppp_orig profile (golden outputs of ScrimpppOrig.cpp).  The
chirped-sine cases have hundreds of windows whose nearest neighbour is exactly
m/4 away, which only PreSCRIMP evaluates; without the merge those windows
would be off by up to a factor of two."""
from __future__ import annotations

import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle.prescrimp import prescrimp
from test_prescrimp_oracle import check_against_reference, golden_rtol

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "thesiscode_b200", "csrc", "host")

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "scrimppp_merge.hpp"

// argv: PL excl pre_d2 pre_idx d2 idx out_d2 out_idx (raw little-endian files)
template <class T> static std::vector<T> load(const char* f, long n) {
    std::vector<T> v(n);
    FILE* p = std::fopen(f, "rb");
    if (!p || std::fread(v.data(), sizeof(T), n, p) != (size_t)n) std::exit(3);
    std::fclose(p);
    return v;
}
template <class T> static void save(const char* f, const std::vector<T>& v) {
    FILE* p = std::fopen(f, "wb");
    if (!p || std::fwrite(v.data(), sizeof(T), v.size(), p) != v.size()) std::exit(4);
    std::fclose(p);
}
int main(int argc, char** argv) {
    if (argc != 9) return 2;
    const long PL = std::atol(argv[1]), excl = std::atol(argv[2]);
    auto pd = load<double>(argv[3], PL);
    auto pi = load<int64_t>(argv[4], PL);
    auto d = load<double>(argv[5], PL);
    auto i = load<int64_t>(argv[6], PL);
    matrix_profile::merge_prescrimp_lag(PL, excl, pd.data(), pi.data(), d.data(), i.data());
    save(argv[7], d);
    save(argv[8], i);
    return 0;
}
"""


@pytest.fixture(scope="module")
def merge_driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("merge")
    src = d / "merge.cpp"
    src.write_text(DRIVER)
    exe = d / "merge"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{HOST}", str(src), "-o", str(exe)], check=True)
    return str(exe)


def merge(driver, tmp, excl, pre, exact):
    PL = pre[0].size
    files = [tmp / f for f in ("pd", "pi", "d", "i", "od", "oi")]
    for f, a, t in zip(files[:4], (pre[0], pre[1], exact[0], exact[1]),
                       ("<f8", "<i8", "<f8", "<i8")):
        f.write_bytes(np.ascontiguousarray(a, dtype=t).tobytes())
    subprocess.run([driver, str(PL), str(excl), *map(str, files)], check=True)
    return (np.frombuffer(files[4].read_bytes(), "<f8").copy(),
            np.frombuffer(files[5].read_bytes(), "<i8").copy())


def test_merged_profile_is_the_reference_scrimppp(merge_driver, oracle, golden_prescrimp, tmp_path):
    for name, c in golden_prescrimp.items():
        x, m, stride = c["x"], int(c["m"]), int(c["stride"])
        pre = prescrimp(x, m, float(stride))
        exact = oracle.selfjoin(x, m)
        d2, idx = merge(merge_driver, tmp_path, m // 4, pre, exact)
        check_against_reference(x, m, d2, idx, c["exact_dist"], c["exact_index"].astype(np.int64),
                                rtol=golden_rtol(name))
        PL = x.size - m + 1
        lag = np.abs(c["exact_index"].astype(np.int64) - np.arange(PL))
        if name.startswith("chirp"):
            # the cases this merge exists for: many neighbours exactly m/4 away
            assert int((lag == m // 4).sum()) > 100
            assert not np.allclose(np.sqrt(np.abs(exact[0])), c["exact_dist"], rtol=1e-3)
