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


def test_run_algorithm_statuses_without_a_device(tmp_path):
    import torch
    series = tmp_path / "x.ascii"
    series.write_text("\n".join(str(v) for v in range(200)))
    out = str(tmp_path / "out.ascii")
    # unknown variant, then an unreadable input: both reported before any device use
    assert mp.run_algorithm("no_such_variant", str(series), out, 16) == mp.MP_ERR_INVALID_ARG
    assert mp.run_algorithm("gpu_vert_blocked_fp64", str(tmp_path / "missing.ascii"), out,
                            16) == mp.MP_ERR_IO
    assert "file" in mp.status_string(mp.MP_ERR_IO)
    if not torch.cuda.is_available():
        assert mp.run_algorithm("gpu_vert_blocked_fp64", str(series), out, 16) == mp.MP_ERR_NO_DEVICE


def test_entry_points_reject_null_arguments():
    import ctypes
    L = mp.load_library()
    buf = (ctypes.c_double * 8)()
    ib = (ctypes.c_int64 * 8)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    q = ctypes.cast(ib, ctypes.c_void_p)
    E = mp.MP_ERR_INVALID_ARG
    assert L.mp_selfjoin(None, p, 8, 4, -1, mp.FP64, 0, 0, 0, 0, p, q, None) == E
    assert L.mp_prescrimp(None, p, 8, 4, 1.0, p, q, None) == E
    assert L.mp_window_stats(None, p, 8, 4, p, p, None) == E
    assert L.mp_first_qt(None, p, 8, 4, 0, 1, p, None) == E
    assert L.mp_eval_diag_block_triangle(None, p, q, p, q, p, 1, 1, p, p, 4, p, p, p, p, 0, 0,
                                         None) == E
    assert L.mp_context_create(0, 0, None) == E
    assert L.mp_context_destroy(None) == E
    assert L.mp_last_error(None) == b"no context"
    assert L.mp_last_launch_count(None) == -1 and L.mp_last_near_duplicates(None) == -1
    assert L.mp_set_phase_timing(None, 1) == E
    srv = ctypes.c_void_p()
    assert L.mp_server_create(0, 0, 1, mp.FP32_REANCHOR, 0, ctypes.byref(srv)) == E  # no budget
    assert L.mp_server_create(0, 1 << 30, 0, mp.FP32_REANCHOR, 0, ctypes.byref(srv)) == E  # no slot
    assert L.mp_server_create(0, 1 << 30, 1, 7, 0, ctypes.byref(srv)) == E  # unknown form
    assert L.mp_server_submit(None, p, 8, 4, ctypes.byref(ctypes.c_int64())) == E
    assert L.mp_batch_create(None, 1, q, q, None, 0, ctypes.byref(srv)) == E
    v = ctypes.c_double()
    assert L.mp_measure_fma_peak(0, 3, ctypes.byref(v)) == E
    assert L.mp_run_algorithm(None, b"x", b"y", 16, 0, 0, 1, 0, 0) == E


def test_allocation_free_entry_checks_arguments_before_the_device():
    import ctypes
    L = mp.load_library()
    L.mp_selfjoin_fp32_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                           ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                           ctypes.c_size_t]
    err = ctypes.create_string_buffer(256)
    fake = ctypes.c_void_p(256)  # never dereferenced: the size checks come first
    rc = L.mp_selfjoin_fp32_noalloc(None, 100, 10, -1, 0, fake, fake, None, err, 256)
    assert rc == mp.MP_ERR_INVALID_ARG and b"null" in err.value
    rc = L.mp_selfjoin_fp32_noalloc(fake, 100, 1, -1, 0, fake, fake, None, err, 256)
    assert rc == mp.MP_ERR_INVALID_ARG and b"window length" in err.value
    rc = L.mp_selfjoin_fp32_noalloc(fake, 5, 10, -1, 0, fake, fake, None, err, 256)
    assert rc == mp.MP_ERR_INVALID_ARG and b"shorter" in err.value
    rc = L.mp_selfjoin_fp32_noalloc(fake, 1 << 20, 10, -1, 0, fake, fake, None, err, 256)
    assert rc == mp.MP_ERR_NOT_SUPPORTED and b"mp_selfjoin" in err.value


def test_cli_accepts_the_reference_options(tmp_path):
    # --dbg (waits for Enter), --dist-io and --chunksize are the reference CLI's; they parse
    # here, and the run then stops only for want of a B200 (or succeeds on one)
    import torch
    x = tmp_path / "x.ascii"
    x.write_text(" ".join(str(float(v)) for v in range(300)))
    r = subprocess.run([mp.CLI_PATH, "gpu_vert_blocked_fp64", "32", "8", str(x), "--dist-io", "false",
                        "--chunksize", "100", "--dbg", "--output-file", str(tmp_path / "o.ascii")],
                       input="\n", capture_output=True, text=True, timeout=120)
    assert "parsing" not in r.stderr and "Press ENTER" in r.stdout
    if not torch.cuda.is_available():
        assert r.returncode == 1 and "no usable device" in r.stderr
    r = subprocess.run([mp.CLI_PATH, "gpu_vert_blocked_fp64", "32", "8", str(x), "--dist-io", "maybe"],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "invalid boolean" in r.stderr


C_PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "mpgpu.h"

int main(void) {
    mp_context* ctx = NULL;
    char names[256];
    int need = mp_list_algorithms(names, sizeof names);
    if (need <= 1 || strstr(names, "gpu_vert_blocked_fp64") == NULL) return 10;
    if (strcmp(mp_status_string(MP_OK), "ok") != 0) return 11;
    if (mp_selfjoin_scratch_bytes(1 << 16, 256, MP_PREC_FP32_REANCHOR) == 0) return 12;
    if (mp_selfjoin(NULL, NULL, 0, 0, -1, MP_PREC_FP64, 0, 0, 0, 0, NULL, NULL, NULL)
        != MP_ERR_INVALID_ARG) return 13;
    {
        const int rc = mp_context_create(0, 0, &ctx);
        printf("%d\n", rc);
        if (rc == MP_OK) mp_context_destroy(ctx);
        else if (rc != MP_ERR_NO_DEVICE) return 14;
    }
    return 0;
}
"""


def test_header_compiles_as_c_and_links(tmp_path):
    # the boundary is plain C: a C99 program includes mpgpu.h and links the library
    import shutil
    import torch
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    src = tmp_path / "use.c"
    src.write_text(C_PROGRAM)
    exe = tmp_path / "use"
    libdir = os.path.dirname(mp.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", f"-I{os.path.join(ROOT, 'include')}",
                    str(src), "-o", str(exe), f"-L{libdir}", "-lmpgpu", f"-Wl,-rpath,{libdir}"],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    if not torch.cuda.is_available():
        assert r.stdout.strip() == str(mp.MP_ERR_NO_DEVICE)
