"""The C-ABI library without a GPU: it loads, exports every function that
include/mpgpu.h declares, and refuses cleanly when no B200 is present."""
from __future__ import annotations

import os
import re
import subprocess

import pytest

import thesiscode_b200 as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mpgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mp_[a-z0-9_]+)\s*\(", text)))


def test_header_and_python_symbol_lists_agree():
    assert declared_functions() == sorted(mp.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = mp.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", mp.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (mp_[a-z0-9_]+)$", out, flags=re.M))
    assert set(declared_functions()) <= exported


def test_status_strings():
    assert mp.status_string(mp.MP_OK) == "ok"
    assert "budget" in mp.status_string(mp.MP_ERR_BUDGET)


def test_registry_lists_gpu_variants():
    names = mp.list_algorithms()
    assert "gpu_vert_blocked_fp64" in names and "gpu_vert_blocked_fp32k" in names
    assert "gpu_scrimppp" in names


def test_scratch_estimate_grows_with_n():
    a = mp.load_library().mp_selfjoin_scratch_bytes(1 << 16, 256, mp.FP32_REANCHOR)
    b = mp.load_library().mp_selfjoin_scratch_bytes(1 << 20, 256, mp.FP32_REANCHOR)
    assert 0 < a < b
    assert mp.load_library().mp_selfjoin_scratch_bytes(10, 20, mp.FP64) == 0


def test_context_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(mp.MpError) as e:
        mp.Context(0)
    assert e.value.status == mp.MP_ERR_NO_DEVICE


def test_cli_help_and_unknown_algorithm():
    r = subprocess.run([mp.CLI_PATH, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "gpu_vert_blocked_fp64" in r.stdout
    r = subprocess.run([mp.CLI_PATH, "no_such_algo", "64", "16", "x.ascii"], capture_output=True,
                       text=True)
    assert r.returncode != 0 and "not known" in r.stderr


def test_cells_count():
    n, m = 65_536, 400
    PL, excl = n - m + 1, m // 4
    assert mp.cells(n, m) == (PL - excl - 1) * (PL - excl) // 2
    assert mp.cells(n, m, 200, 300) == sum(PL - d for d in range(200, 300))
