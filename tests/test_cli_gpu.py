"""The drop-in command line and file formats on the GPU: mpgpu_cli with the
reference's arguments must write the same ASCII profile file as the
reference's own binary, byte for byte, and read/write the binary formats."""
from __future__ import annotations

import hashlib
import os
import subprocess

import numpy as np
import pytest

import thesiscode_b200 as mp

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _write_ascii(path, x):
    with open(path, "w") as f:
        f.write(" ".join(repr(float(v)) for v in x))


def test_cli_ascii_matches_reference_file(tmp_path, golden_ascii):
    inp = tmp_path / "test.ascii"
    _write_ascii(inp, golden_ascii["series"])
    out = tmp_path / "prof.ascii"
    r = subprocess.run([mp.CLI_PATH, "gpu_vert_blocked_fp64", "400", "100", str(inp),
                        "--output-file", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    text = out.read_text()
    head = open(os.path.join(HERE, "golden", "ascii_cli_m400.txt")).read().splitlines()
    want_sha = head[0].split()[2]
    assert hashlib.sha256(text.encode()).hexdigest() == want_sha
    assert text.splitlines()[:40] == head[1:41]


def test_cli_default_output_name(tmp_path, golden_ascii):
    inp = tmp_path / "series.ascii"
    _write_ascii(inp, golden_ascii["series"][:3000])
    r = subprocess.run([mp.CLI_PATH, "gpu_vert_blocked_fp32k", "64", "16", str(inp)],
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "gpu_vert_blocked_fp32k_new_MatrixProfile_64series.ascii.matprof.ascii").exists()


def test_cli_binary_round_trip(tmp_path, golden_ascii, digests):
    x = golden_ascii["series"]
    hdr = np.zeros(100, dtype=np.uint8)
    hdr[:16] = np.frombuffer(np.array([2, 100], dtype="<u4").tobytes()
                             + np.array([x.size], dtype="<u8").tobytes(), dtype=np.uint8)
    inp = tmp_path / "test.bin"
    inp.write_bytes(hdr.tobytes() + x.astype("<f8").tobytes())
    out = tmp_path / "prof.bin"
    r = subprocess.run([mp.CLI_PATH, "gpu_vert_blocked_fp64", "64", "16", str(inp),
                        "--output-file", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    b = out.read_bytes()
    fmt, off = np.frombuffer(b[:8], "<u4")
    count = int(np.frombuffer(b[8:16], "<u8")[0])
    assert (fmt, off, count) == (1, 100, x.size - 64 + 1)
    rec = np.frombuffer(b[100:], dtype=[("d2", "<f8"), ("idx", "<u8")])
    assert np.array_equal(rec["d2"], golden_ascii["d2_m64"])  # binary stores d2, not sqrt
    assert np.array_equal(rec["idx"].astype(np.int64), golden_ascii["idx_m64"])
    # the input is the reference's test.bin and the output the file its own MPI-IO
    # writer makes for it, byte for byte
    assert hashlib.sha256(inp.read_bytes()).hexdigest() == digests["test_bin"]["sha256"]
    assert hashlib.sha256(b).hexdigest() == digests["bin_profile_test_bin_m64"]["sha256"]


def test_run_algorithm_through_registry(tmp_path, golden_ascii):
    inp = tmp_path / "s.ascii"
    _write_ascii(inp, golden_ascii["series"])
    out = tmp_path / "p.ascii"
    assert mp.run_algorithm("gpu_vert_blocked_fp64", str(inp), str(out), 16) == mp.MP_OK
    got = np.loadtxt(out)
    assert np.array_equal(got[:, 1].astype(np.int64), golden_ascii["idx_m16"])
    assert mp.run_algorithm("no_such_variant", str(inp), str(out), 16) == mp.MP_ERR_INVALID_ARG


def test_cli_outputs_pass_the_validation_tool(tmp_path, golden_ascii):
    """The reference's validation workflow on the drop-in CLI's files: the FP64
    variant's profile coincides with the reference's profile; the FP32
    variant's indices agree up to neighbours whose distances tie within 1e-4."""
    from thesiscode_b200 import validate
    x = golden_ascii["series"]
    inp = tmp_path / "test.ascii"
    _write_ascii(inp, x)
    ref = tmp_path / "ref.ascii"
    validate.write_profile_ascii(str(ref), golden_ascii["d2_m64"], golden_ascii["idx_m64"])
    outs = {}
    for algo in ("gpu_vert_blocked_fp64", "gpu_vert_blocked_fp32k"):
        outs[algo] = tmp_path / f"{algo}.matprof.ascii"
        r = subprocess.run([mp.CLI_PATH, algo, "64", "16", str(inp),
                            "--output-file", str(outs[algo])], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    assert validate.main(["compare", str(ref), str(outs["gpu_vert_blocked_fp64"]),
                          "--silent"]) == 0
    assert validate.main(["compare", str(outs["gpu_vert_blocked_fp64"]),
                          str(outs["gpu_vert_blocked_fp32k"]), "--silent", "--series", str(inp),
                          "--window", "64", "--rel-tol", "1e-4"]) == 0
