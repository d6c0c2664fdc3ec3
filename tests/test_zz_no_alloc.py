"""The allocation-free self-join, mp_selfjoin_fp32_noalloc, called through the
C-ABI with device buffers the test owns.

It exists for callers that cannot allocate device memory (a framework that owns
the GPU through its own pool, or a path where cudaMalloc's implicit
synchronisation is not allowed).  Its results must match mp_selfjoin's FP32
form with the same re-anchor interval, within the FP32 tolerance used across
these tests (1e-4 relative distance), on consecutive calls that reuse the one
static scratch array: the second call is shorter than the first, so anything
the first call left behind would show up in it.  The file is named to be
collected last."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import thesiscode_b200 as mp

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4
MP_ERR_NOT_SUPPORTED = 5
MAX_N = 131072  # MPGPU_NOALLOC_MAX_N in include/mpgpu.h


def _entry():
    lib = ctypes.CDLL(mp.LIB_PATH)
    f = lib.mp_selfjoin_fp32_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                  ctypes.c_size_t]
    return f


def _series(seed, n):
    rng = np.random.default_rng(seed)
    x = np.cumsum(rng.standard_normal(n))
    x[n // 3: n // 3 + 500] = 1.5  # a flat stretch: its windows have no neighbour
    return x


def _buffers(torch, x, m):
    A = torch.from_numpy(x).cuda()
    PL = x.size - m + 1
    d2 = torch.full((PL,), -1.0, dtype=torch.float64, device="cuda")
    ix = torch.full((PL,), -1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    return A, d2, ix


def _call(f, torch, bufs, n, m, k, excl=-1):
    A, d2, ix = bufs
    err = ctypes.create_string_buffer(256)
    rc = f(A.data_ptr(), n, m, excl, k, d2.data_ptr(), ix.data_ptr(),
           torch.cuda.current_stream().cuda_stream, err, len(err))
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    return d2.cpu().numpy(), ix.cpu().numpy()


def _noalloc(f, torch, x, m, k, excl=-1):
    return _call(f, torch, _buffers(torch, x, m), x.size, m, k, excl)


def _check_same(got, want):
    d2, ix = got
    a, b = np.sqrt(np.abs(d2)), np.sqrt(np.abs(want.dist2))
    rel = np.abs(a - b) / np.maximum(b, 1e-12)
    assert rel.max() <= REL_TOL, rel.max()
    assert np.array_equal(ix, want.index)


def test_noalloc_matches_selfjoin_on_consecutive_calls(gpu_ctx):
    import torch
    f = _entry()
    cases = [(_series(11, MAX_N), 256, 512), (_series(12, 7000), 32, 0)]
    want = [gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=k) for x, m, k in cases]
    for (x, m, k), w in zip(cases, want):
        _check_same(_noalloc(f, torch, x, m, k), w)
    # and the long case once more, after the short one has used the scratch
    x, m, k = cases[0]
    _check_same(_noalloc(f, torch, x, m, k), want[0])


def test_noalloc_rejects_series_beyond_limit():
    import torch
    f = _entry()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    err = ctypes.create_string_buffer(256)
    rc = f(buf.data_ptr(), MAX_N + 1, 64, -1, 0, buf.data_ptr(), buf.data_ptr(), None, err,
           len(err))
    assert rc == MP_ERR_NOT_SUPPORTED
    assert b"allocation-free limit" in err.value


def test_noalloc_allocates_nothing(gpu_ctx):
    """After a first call (which only looks up the scratch address), further
    calls leave the device's free memory and torch's allocator untouched."""
    import torch
    f = _entry()
    x, m, k = _series(13, 50_000), 128, 1024
    bufs = _buffers(torch, x, m)
    first = _call(f, torch, bufs, x.size, m, k)
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    again = [_call(f, torch, bufs, x.size, m, k) for _ in range(2)]
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0
    assert free1 == free0
    for d2, ix in again:
        assert np.array_equal(d2, first[0]) and np.array_equal(ix, first[1])


@pytest.mark.parametrize("excl", [20, 9000])
def test_noalloc_explicit_exclusion_zone(gpu_ctx, excl):
    """An explicit exclusion zone, and one at least as long as the profile (no
    diagonal is evaluated, so every window keeps the no-neighbour result)."""
    import torch
    f = _entry()
    x, m, k = _series(14, 9000), 64, 256
    want = gpu_ctx.selfjoin(x, m, precision=mp.FP32_REANCHOR, reanchor_k=k, excl=excl)
    _check_same(_noalloc(f, torch, x, m, k, excl=excl), want)
    if excl >= x.size - m + 1:
        assert np.all(want.dist2 == 2 * m + 2)


def test_noalloc_refuses_buffers_of_another_gpu():
    """A buffer on another GPU is refused before anything is launched."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    f = _entry()
    other = torch.zeros(4096, dtype=torch.float64, device="cuda:1")
    mine = torch.zeros(4096, dtype=torch.float64, device="cuda:0")
    torch.cuda.set_device(0)
    err = ctypes.create_string_buffer(256)
    rc = f(other.data_ptr(), 4096, 64, -1, 0, mine.data_ptr(), mine.data_ptr(), None, err,
           len(err))
    assert rc == mp.MP_ERR_INVALID_ARG
    assert b"current device" in err.value
