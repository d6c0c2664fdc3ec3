"""The C++ series/profile file layer (thesiscode_b200/csrc/host/profile_io.cpp)
on CPU: compiled with g++ into a small driver, checked against the Python
readers/writers of thesiscode_b200/validate.py and against hand-built files in
the reference's formats (100-byte header {u32 format, u32 offset, u64 count};
format 2 = series of doubles, format 1 = {double d2, u64 index}; ASCII profile =
sqrt(|d2|) with 17 significant digits).  Truncated or corrupt headers must give
an error message, not an allocation of the header's count."""
from __future__ import annotations

import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from thesiscode_b200 import validate

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "thesiscode_b200", "csrc", "host")

DRIVER = r"""
#include "profile_io.hpp"
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>
using namespace matrix_profile::io;

static void print(const std::vector<double>& d, const std::vector<int64_t>* idx) {
    std::printf("%zu\n", d.size());
    for (size_t i = 0; i < d.size(); ++i) {
        if (idx) std::printf("%.17g %lld\n", d[i], (long long)(*idx)[i]);
        else std::printf("%.17g\n", d[i]);
    }
}

int main(int argc, char** argv) {
    const std::string cmd = argv[1], path = argv[2];
    try {
        if (cmd == "read_series_bin") print(read_series_bin(path), nullptr);
        else if (cmd == "read_series_ascii") print(read_series_ascii(path), nullptr);
        else if (cmd == "read_profile_bin") {
            std::vector<double> d2;
            std::vector<int64_t> idx;
            read_profile_bin(path, d2, idx);
            print(d2, &idx);
        } else {  // write_*: values from stdin, "n" then n lines "d2 index"
            long long n = 0;
            if (std::scanf("%lld", &n) != 1) return 2;
            std::vector<double> d2(n);
            std::vector<int64_t> idx(n);
            for (long long i = 0; i < n; ++i) {
                long long k = 0;
                if (std::scanf("%lf %lld", &d2[i], &k) != 2) return 2;
                idx[i] = k;
            }
            if (cmd == "write_series_bin") write_series_bin(path, d2);
            else if (cmd == "write_profile_bin") write_profile_bin(path, d2.data(), idx.data(), n);
            else if (cmd == "write_profile_ascii") write_profile_ascii(path, d2.data(), idx.data(), n);
            else return 2;
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ERROR: %s\n", e.what());
        return 1;
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("pio")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "pio"
    subprocess.run(["g++", "-std=c++17", "-O1", f"-I{HOST}", str(src), os.path.join(HOST, "profile_io.cpp"),
                    "-o", str(exe)], check=True)
    return str(exe)


def _run(driver, *args, stdin=None):
    return subprocess.run([driver, *args], input=stdin, capture_output=True, text=True)


def _values(out: str):
    lines = out.split("\n")
    n = int(lines[0])
    rows = [ln.split() for ln in lines[1:1 + n]]
    return n, rows


def _stdin(d2, idx):
    # repr() of a float round-trips exactly through scanf("%lf")
    return f"{len(d2)}\n" + "".join(f"{float(v)!r} {int(i)}\n" for v, i in zip(d2, idx))


def test_series_bin_read_and_write(driver, tmp_path):
    x = np.cumsum(np.random.default_rng(1).standard_normal(1000))
    f = tmp_path / "s.bin"
    f.write_bytes(struct.pack("<IIQ", 2, 100, x.size).ljust(100, b"\0") + x.astype("<f8").tobytes())
    r = _run(driver, "read_series_bin", str(f))
    assert r.returncode == 0, r.stderr
    n, rows = _values(r.stdout)
    assert n == x.size and np.array_equal(np.array([float(v[0]) for v in rows]), x)
    g = tmp_path / "w.bin"
    r = _run(driver, "write_series_bin", str(g), stdin=_stdin(x, np.zeros(x.size)))
    assert r.returncode == 0, r.stderr
    raw = g.read_bytes()
    assert struct.unpack("<IIQ", raw[:16]) == (2, 100, x.size) and raw[16:100] == b"\0" * 84
    assert np.array_equal(np.frombuffer(raw[100:], "<f8"), x)
    assert np.array_equal(validate.read_series(str(g)), x)


def test_profile_bin_round_trip_with_python(driver, tmp_path):
    rng = np.random.default_rng(2)
    d2 = rng.uniform(0, 500, 777)
    idx = rng.integers(0, 1 << 40, 777)
    f = tmp_path / "p.bin"
    r = _run(driver, "write_profile_bin", str(f), stdin=_stdin(d2, idx))
    assert r.returncode == 0, r.stderr
    raw = f.read_bytes()
    assert struct.unpack("<IIQ", raw[:16]) == (1, 100, d2.size) and raw[16:100] == b"\0" * 84
    rec = np.frombuffer(raw[100:], dtype=[("d2", "<f8"), ("idx", "<u8")])
    assert np.array_equal(rec["d2"], d2) and np.array_equal(rec["idx"].astype(np.int64), idx)
    dist, pidx = validate.read_profile(str(f))  # the reader gives distances, sqrt(|d2|)
    assert np.array_equal(dist, np.sqrt(d2)) and np.array_equal(pidx, idx)
    g = tmp_path / "q.bin"
    validate.write_profile_bin(str(g), d2, idx)
    r = _run(driver, "read_profile_bin", str(g))
    assert r.returncode == 0, r.stderr
    n, rows = _values(r.stdout)
    assert n == d2.size
    assert np.array_equal(np.array([float(v[0]) for v in rows]), d2)
    assert np.array_equal(np.array([int(v[1]) for v in rows]), idx)


def test_profile_ascii_holds_the_root_with_17_digits(driver, tmp_path):
    d2 = np.array([0.0, 2.5, 1e-300, 513.0, -1e-12])
    idx = np.array([0, 7, 3, 12345678901, 2])
    f = tmp_path / "p.ascii"
    r = _run(driver, "write_profile_ascii", str(f), stdin=_stdin(d2, idx))
    assert r.returncode == 0, r.stderr
    rows = [ln.split() for ln in f.read_text().splitlines()]
    assert np.array_equal(np.array([float(a) for a, _ in rows]), np.sqrt(np.abs(d2)))
    assert [int(b) for _, b in rows] == list(idx)


def test_series_ascii_reads_whitespace_separated(driver, tmp_path):
    f = tmp_path / "s.ascii"
    f.write_text("1.5 -2\n3e2\t4.25\n\n5\n")
    r = _run(driver, "read_series_ascii", str(f))
    assert r.returncode == 0, r.stderr
    n, rows = _values(r.stdout)
    assert n == 5 and [float(v[0]) for v in rows] == [1.5, -2.0, 300.0, 4.25, 5.0]


@pytest.mark.parametrize("count", [11, 1 << 60])
def test_truncated_or_corrupt_counts_are_errors(driver, tmp_path, count):
    f = tmp_path / "s.bin"
    f.write_bytes(struct.pack("<IIQ", 2, 100, count).ljust(100, b"\0") + np.zeros(10).tobytes())
    r = _run(driver, "read_series_bin", str(f))
    assert r.returncode == 1 and "truncated series file" in r.stderr, r.stderr
    g = tmp_path / "p.bin"
    g.write_bytes(struct.pack("<IIQ", 1, 100, count).ljust(100, b"\0") + np.zeros(20).tobytes())
    r = _run(driver, "read_profile_bin", str(g))
    assert r.returncode == 1 and "truncated profile file" in r.stderr, r.stderr
    for path in (f, g):  # the Python readers refuse them too
        with pytest.raises(ValueError, match="truncated"):
            (validate.read_series if path is f else validate.read_profile)(str(path))


def test_wrong_format_or_offset_is_an_error(driver, tmp_path):
    f = tmp_path / "s.bin"
    f.write_bytes(struct.pack("<IIQ", 1, 100, 2).ljust(100, b"\0") + np.zeros(2).tobytes())
    r = _run(driver, "read_series_bin", str(f))
    assert r.returncode == 1 and "unexpected binary format 1" in r.stderr
    f.write_bytes(struct.pack("<IIQ", 2, 64, 2).ljust(100, b"\0") + np.zeros(2).tobytes())
    r = _run(driver, "read_series_bin", str(f))
    assert r.returncode == 1 and "unexpected data offset" in r.stderr
    r = _run(driver, "read_series_bin", str(tmp_path / "missing.bin"))
    assert r.returncode == 1 and "Could not open input file" in r.stderr


def test_writer_reproduces_the_reference_binary_series_file(driver, tmp_path, golden_ascii, digests):
    # the reference ships test.ascii and its binary copy test.bin (format 2);
    # written from test.ascii's values, our file must be that file byte for byte
    import hashlib
    x = golden_ascii["series"]
    g = tmp_path / "test.bin"
    r = _run(driver, "write_series_bin", str(g), stdin=_stdin(x, np.zeros(x.size)))
    assert r.returncode == 0, r.stderr
    raw = g.read_bytes()
    assert len(raw) == digests["test_bin"]["bytes"]
    assert hashlib.sha256(raw).hexdigest() == digests["test_bin"]["sha256"]
    r = _run(driver, "read_series_bin", str(g))
    assert r.returncode == 0 and _values(r.stdout)[0] == x.size
    assert np.array_equal(validate.read_series(str(g)), x)


def test_writer_reproduces_the_reference_binary_profile_file(driver, tmp_path, golden_ascii, digests):
    # the reference's MPI-IO profile writer (binproffile.cpp, run for its test.bin with
    # m = 64) made a file with this digest; ours, given the same profile, must match
    import hashlib
    d2, idx = golden_ascii["d2_m64"], golden_ascii["idx_m64"]
    g = tmp_path / "prof.bin"
    r = _run(driver, "write_profile_bin", str(g), stdin=_stdin(d2, idx))
    assert r.returncode == 0, r.stderr
    raw = g.read_bytes()
    assert len(raw) == digests["bin_profile_test_bin_m64"]["bytes"]
    assert hashlib.sha256(raw).hexdigest() == digests["bin_profile_test_bin_m64"]["sha256"]



@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "scrimppp_ref_bin")),
                    reason="oracle/_ref not built (no reference tree)")
def test_files_interchange_with_the_reference(driver, tmp_path, oracle):
    # our series file goes into the reference's binary reader; the reference's binary
    # profile comes back through our reader
    from thesiscode_b200 import workloads
    x, m = workloads.random_walk(1500, 11), 40
    s = tmp_path / "series.bin"
    r = _run(driver, "write_series_bin", str(s), stdin=_stdin(x, np.zeros(x.size)))
    assert r.returncode == 0, r.stderr
    p = tmp_path / "prof.bin"
    ref = os.path.join(ROOT, "oracle", "_ref", "scrimppp_ref_bin")
    subprocess.run([ref, "scrimp_vert_blocked", str(m), "1", str(s), "--filetype", "BIN",
                    "--output-file", str(p)], check=True, capture_output=True)
    r = _run(driver, "read_profile_bin", str(p))
    assert r.returncode == 0, r.stderr
    n, rows = _values(r.stdout)
    d2, idx = oracle.selfjoin(x, m)
    assert n == d2.size
    assert np.array_equal(np.array([float(v[0]) for v in rows]), d2)
    assert np.array_equal(np.array([int(v[1]) for v in rows]), idx)
