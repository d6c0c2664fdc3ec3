"""Regenerates the golden fixtures in this directory from the REFERENCE itself.

Run in a container where the reference tree exists (it is read at build time
only): ``SCRIMP_REF_ROOT=<reference checkout>/scrimppp python
tests/golden/make_golden.py [--big]``.  It builds
oracle/_ref from the reference's unchanged sources (oracle/Makefile) and
records what those binaries output:

  test_ascii.npz     the reference's own fixture scrimppp/data_testing/test.ascii
                     (10,000 samples) and, for m in {16, 64, 400}, the
                     profile (squared distance) and index of scrimp_vert_blocked
                     (IEEE build, shuffled block order as the reference runs it),
                     its window statistics and first dot products for m = 64
  ascii_cli_m400.txt head of the reference CLI's ASCII output for
                     test.ascii, m = 400, plus the sha256 of the whole file
  edge_cases.npz     small seeded cases: tiny series, blocklen not a multiple
                     of 4, zero- and non-zero-level flat segments, n == m,
                     a single diagonal, odd m, a large offset
  digests.json       sha256 of the reference's own binary copy of test.ascii
                     (data_testing/test.bin, series format 2); of the binary
                     profile (format 1) the reference's MPI-IO classes write
                     for test.bin with m = 64 (oracle/_ref/scrimppp_ref_bin,
                     --filetype BIN); and
                     sha256 of the reference's d2/idx bytes for workload c1
                     (n = 65,536, m = 400), and with --big for c2
                     (n = 1,048,576, m = 256, values from the threaded triv_par
                     re-hosting; indices may only differ on exact ties)
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import REF_SRC, RefOracle, build  # noqa: E402
from thesiscode_b200 import workloads  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def edge_cases():
    rng = np.random.default_rng(12345)
    cases = {}

    def add(name, x, m, B=500):
        cases[name] = (np.asarray(x, dtype=np.float64), m, B)

    add("tiny_m8", np.cumsum(rng.standard_normal(200)), 8)
    add("tiny_m8_B7", np.cumsum(rng.standard_normal(200)), 8, 7)
    add("n300_m16_B1", np.cumsum(rng.standard_normal(300)), 16, 1)
    add("n300_m16_B3", np.cumsum(rng.standard_normal(300)), 16, 3)
    add("n300_m16_B13", np.cumsum(rng.standard_normal(300)), 16, 13)
    x = np.cumsum(rng.standard_normal(2000))
    x[500:700] = 0.0
    add("flat_zero_level", x, 64)
    x = np.cumsum(rng.standard_normal(2000))
    x[1200:1400] = 7.25
    add("flat_nonzero_level", x, 64)
    add("n_equals_m", np.cumsum(rng.standard_normal(32)), 32)
    add("single_diagonal", np.cumsum(rng.standard_normal(16 + 4 + 1)), 16)
    add("odd_m37", np.cumsum(rng.standard_normal(1500)), 37)
    add("offset_1e4", 1.0e4 + np.cumsum(rng.standard_normal(1500)), 50)
    add("white_noise", rng.standard_normal(3000), 100, 64)
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true", help="also digest workload c2 (minutes)")
    args = ap.parse_args()
    build(with_reference=True)
    ieee = RefOracle("ieee")
    fast = RefOracle("fast")

    series = np.array(open(os.path.join(REF_SRC, "data_testing", "test.ascii")).read().split(),
                      dtype=np.float64)
    out = {"series": series}
    for m in (16, 64, 400):
        d2, idx, _ = ieee.vert_blocked(series, m, shuffle=True)
        out[f"d2_m{m}"] = d2
        out[f"idx_m{m}"] = idx
        d2f, idxf, _ = fast.vert_blocked(series, m, shuffle=True)
        out[f"fast_maxrel_m{m}"] = np.array(
            np.max(np.abs(np.sqrt(np.abs(d2f)) - np.sqrt(np.abs(d2))) / np.sqrt(np.abs(d2))))
        out[f"fast_idxdiff_m{m}"] = np.array((idxf != idx).sum())
    muS, sInv = ieee.window_stats(series, 64)
    out["muS_m64"] = muS
    out["sInv_m64"] = sInv
    out["qt_m64_0_2000"] = ieee.first_qt(series, 64, 0, 1999)
    np.savez_compressed(os.path.join(HERE, "test_ascii.npz"), **out)

    with tempfile.TemporaryDirectory() as td:
        of = os.path.join(td, "out.ascii")
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "scrimppp_ref_ieee"),
                        "scrimp_vert_blocked", "400", "100",
                        os.path.join(REF_SRC, "data_testing", "test.ascii"),
                        "--output-file", of], check=True, capture_output=True)
        text = open(of).read()
        head = "".join(text.splitlines(keepends=True)[:40])
        with open(os.path.join(HERE, "ascii_cli_m400.txt"), "w") as f:
            f.write(f"# sha256 {hashlib.sha256(text.encode()).hexdigest()} "
                    f"lines {text.count(chr(10))}\n")
            f.write(head)

    ec = {}
    for name, (x, m, B) in edge_cases().items():
        d2, idx, _ = ieee.vert_blocked(x, m, blocklen=B, shuffle=True)
        ec[f"{name}__x"] = x
        ec[f"{name}__meta"] = np.array([m, B])
        ec[f"{name}__d2"] = d2
        ec[f"{name}__idx"] = idx
    np.savez_compressed(os.path.join(HERE, "edge_cases.npz"), **ec)

    dig = {}
    tb = open(os.path.join(REF_SRC, "data_testing", "test.bin"), "rb").read()
    dig["test_bin"] = {"bytes": len(tb), "sha256": hashlib.sha256(tb).hexdigest()}
    with tempfile.TemporaryDirectory() as td:
        of = os.path.join(td, "prof.bin")
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "scrimppp_ref_bin"),
                        "scrimp_vert_blocked", "64", "1",
                        os.path.join(REF_SRC, "data_testing", "test.bin"),
                        "--filetype", "BIN", "--output-file", of], check=True, capture_output=True)
        pb = open(of, "rb").read()
    rec = np.frombuffer(pb[100:], dtype=[("d2", "<f8"), ("idx", "<u8")])
    assert np.array_equal(rec["d2"], out["d2_m64"])  # the binary read gave the same series
    dig["bin_profile_test_bin_m64"] = {"bytes": len(pb), "sha256": hashlib.sha256(pb).hexdigest()}
    x, m = workloads.c1()
    d2, idx, sec = ieee.vert_blocked(x, m, shuffle=True)
    dig["c1"] = {"n": int(x.size), "m": m, "d2_sha256": sha(d2), "idx_sha256": sha(idx),
                 "d2_min": float(d2.min()), "d2_mean": float(d2.mean()),
                 "ref_seconds_1core": sec}
    if args.big:
        x, m = workloads.c2()
        PL = x.size - m + 1
        d2, idx, sec = ieee.triv_par_threads(x, m, m // 4 + 1, PL, os.cpu_count() or 8)
        dig["c2"] = {"n": int(x.size), "m": m, "d2_sha256": sha(d2), "idx_sha256": sha(idx),
                     "d2_min": float(d2.min()), "d2_mean": float(d2.mean()),
                     "ref_seconds": sec, "ref_threads": os.cpu_count()}
    else:
        old = os.path.join(HERE, "digests.json")
        if os.path.exists(old):
            prev = json.load(open(old))
            if "c2" in prev:
                dig["c2"] = prev["c2"]
    json.dump(dig, open(os.path.join(HERE, "digests.json"), "w"), indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
