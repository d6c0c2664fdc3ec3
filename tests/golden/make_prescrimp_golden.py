"""Regenerates tests/golden/prescrimp_ref.npz from the REFERENCE's PreSCRIMP.

Run where the reference tree exists: ``SCRIMP_REF_ROOT=<reference checkout>/scrimppp
python tests/golden/make_prescrimp_golden.py``.
It builds oracle/_ref/scrimppp_ref_orig (oracle/Makefile: the reference's
ScrimpppOrig.cpp and the hot-path sources, unchanged, IEEE build, with the
stand-in FFT of oracle/ref_fftw_stub.cpp in place of FFTW), runs the
reference's ``scrimppp_orig`` variant through its factory on each case below
and records the ``<output>_prescrimp`` file it writes
(ScrimpppOrig.cpp:275-283): per window sqrt(|d2|) printed with 17 significant
digits (an exact double round trip) and the neighbour index; and the final
``<output>`` file (:388-392), the SCRIMP phase's exact diagonals lowering the
PreSCRIMP profile, as ``exact_dist``/``exact_index``.

Cases (seeded; series stored in the fixture): random walks with power-of-two
and other FFT sizes, an odd window, white noise, a large offset, strides 1, 2
and 5 (the reference's stride is an integer multiple of the window), and the
smallest series, where the FFT size is 2m instead of n
(ScrimpppOrig.cpp:127-128), and slowly chirped sines of period m/4, whose
nearest neighbours lie exactly m/4 away: PreSCRIMP accepts that lag, the exact
diagonals start one further; and the reference README's example
(scrimppp_orig 400 100 on its own data_testing/test.ascii).  No flat windows: there the reference divides
FFT rounding noise by a zero standard deviation, so its result depends on
FFTW's exact rounding.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import REF_DIR, REF_SRC, build  # noqa: E402

BINARY = os.path.join(REF_DIR, "scrimppp_ref_orig")


def cases():
    rng = np.random.default_rng(20240611)
    walk = lambda n: np.cumsum(rng.standard_normal(n))  # noqa: E731
    return [
        ("walk_n2048_m64_s1", walk(2048), 64, 1),
        ("walk_n1500_m50_s1", walk(1500), 50, 1),
        ("walk_n2048_m32_s2", walk(2048), 32, 2),
        ("noise_n2000_m37_s1", rng.standard_normal(2000), 37, 1),
        ("offset_n1024_m16_s3", 1.0e4 + walk(1024), 16, 3),
        ("walk_n1000_m20_s5", walk(1000), 20, 5),
        ("walk_n128_m64_s1", walk(128), 64, 1),
        ("walk_n100_m64_s1", walk(100), 64, 1),
        ("chirp_n2048_m64_s1", chirp(2048, 64, 2e-6, 1e-3, rng), 64, 1),
        ("chirp_n2000_m40_s2", chirp(2000, 40, 1e-5, 1e-3, rng), 40, 2),
        # the reference README's example, scrimppp_orig 400 100 on its test.ascii: one
        # query, whose walk runs the whole length of its best diagonal
        ("readme_test_ascii_m400_s100", test_ascii(), 400, 100),
    ]


def test_ascii():
    return np.array(open(os.path.join(REF_SRC, "data_testing", "test.ascii")).read().split(),
                    dtype=np.float64)


def chirp(n, m, alpha, eps, rng):
    """sin(2 pi t / (m/4) + alpha t^2) plus eps N(0, 1) noise."""
    t = np.arange(n)
    return np.sin(2 * np.pi * t / (m // 4) + alpha * t * t) + eps * rng.standard_normal(n)


def run_reference_both(x: np.ndarray, m: int, stride: int):
    """The reference SCRIMP++'s two profiles of x, each (sqrt(|d2|), index):
    PreSCRIMP's and the final one."""
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "series.ascii")
        out = os.path.join(td, "profile")
        np.savetxt(src, x, fmt="%.17g")
        subprocess.run([BINARY, "scrimppp_orig", str(m), str(stride), src, "--output-file", out],
                       check=True, capture_output=True)
        a = np.loadtxt(out + "_prescrimp", ndmin=2)
        b = np.loadtxt(out, ndmin=2)
    return ((a[:, 0].copy(), a[:, 1].astype(np.int64)),
            (b[:, 0].copy(), b[:, 1].astype(np.int64)))


def run_reference(x: np.ndarray, m: int, stride: int) -> tuple[np.ndarray, np.ndarray]:
    """The reference's PreSCRIMP profile of x: (sqrt(|d2|), index)."""
    return run_reference_both(x, m, stride)[0]


def main():
    build(with_reference=True)
    out = {}
    names = []
    for name, x, m, stride in cases():
        (d, idx), (de, ie) = run_reference_both(x, m, stride)
        assert d.size == x.size - m + 1 == de.size
        out[f"{name}/x"] = x
        out[f"{name}/m"] = np.int64(m)
        out[f"{name}/stride"] = np.int64(stride)
        out[f"{name}/dist"] = d
        out[f"{name}/index"] = idx.astype(np.int32)
        out[f"{name}/exact_dist"] = de
        out[f"{name}/exact_index"] = ie.astype(np.int32)
        names.append(name)
        print(f"{name}: {d.size} windows, min distance {d.min():.6g}")
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "prescrimp_ref.npz"), **out)


if __name__ == "__main__":
    main()
