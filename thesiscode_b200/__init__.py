"""thesiscode_b200 -- B200-native matrix-profile self-join.

Python front end of the in-tree C-ABI library ``libmpgpu.so``
(include/mpgpu.h).  The kernels are hand-written CUDA for sm_100a; this
module only moves arguments across the C boundary.  There is no CPU fallback:
every call that needs the library fails loudly when it is missing or when no
B200 is present.

The names mirror the reference's interface (4rchangel/ThesisCode, scrimppp/):
``selfjoin`` is ScrimpVertBlocked::compute_matrix_profile without file I/O,
``eval_diag_block_triangle`` is the reference kernel (inc/kernels.h:7-24),
``window_stats``/``first_qt`` are ScrimpSequOpt's helpers, and
``list_algorithms``/``run_algorithm`` drive the algorithm-variant factory
(inc/MatProfAlgo.hpp) through the C++ host layer.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpgpu.so")
CLI_PATH = os.path.join(HERE, "mpgpu_cli")

MP_OK = 0
MP_ERR_INVALID_ARG = 1
MP_ERR_OUT_OF_MEMORY = 2
MP_ERR_BUDGET = 3
MP_ERR_CUDA = 4
MP_ERR_NOT_SUPPORTED = 5
MP_ERR_NO_DEVICE = 6
MP_ERR_IO = 7

FP64 = 0
FP32_REANCHOR = 1
FP32_GUARDED = 2  # FP32 re-anchored with FP64 tiles around ill-conditioned windows

FILETYPE_ASCII = 1
FILETYPE_BIN = 2

# Every extern "C" symbol include/mpgpu.h declares.
EXPORTED_SYMBOLS = (
    "mp_context_create", "mp_context_destroy", "mp_last_error", "mp_status_string",
    "mp_selfjoin_scratch_bytes", "mp_selfjoin", "mp_eval_diag_block_triangle",
    "mp_window_stats", "mp_first_qt", "mp_last_launch_count", "mp_list_algorithms",
    "mp_run_algorithm", "mp_set_phase_timing", "mp_last_phase_ms", "mp_measure_fma_peak",
    "mp_batch_create", "mp_batch_destroy", "mp_batch_cells", "mp_batch_tiles",
    "mp_batch_launch_count", "mp_batch_upload", "mp_batch_launch", "mp_batch_download",
    "mp_batch_run", "mp_server_create", "mp_server_submit", "mp_server_poll", "mp_server_collect",
    "mp_server_stats", "mp_server_destroy", "mp_selfjoin_fp32_noalloc", "mp_prescrimp",
    "mp_last_near_duplicates", "mp_selfjoin_ranges",
)


class MpError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


_lib = None
_P = ctypes.c_void_p
_i64 = ctypes.c_int64


def load_library() -> ctypes.CDLL:
    """Loads libmpgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is missing; build it with `python -m thesiscode_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    L.mp_context_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_P)]
    L.mp_context_destroy.argtypes = [_P]
    L.mp_last_error.argtypes = [_P]
    L.mp_last_error.restype = ctypes.c_char_p
    L.mp_status_string.argtypes = [ctypes.c_int]
    L.mp_status_string.restype = ctypes.c_char_p
    L.mp_selfjoin_scratch_bytes.argtypes = [_i64, _i64, ctypes.c_int]
    L.mp_selfjoin_scratch_bytes.restype = ctypes.c_size_t
    L.mp_selfjoin.argtypes = [_P, _P, _i64, _i64, _i64, ctypes.c_int, _i64, _i64, _i64, _i64,
                              _P, _P, _P]
    L.mp_selfjoin_ranges.argtypes = [_P, _P, _i64, _i64, _i64, ctypes.c_int, _i64, _i64, _P,
                                     _i64, _P, _P, _P]
    L.mp_eval_diag_block_triangle.argtypes = [_P, _P, _P, _P, _P, _P, _i64, _i64, _P, _P, _i64,
                                              _P, _P, _P, _P, _i64, _i64, _P]
    L.mp_window_stats.argtypes = [_P, _P, _i64, _i64, _P, _P, _P]
    L.mp_first_qt.argtypes = [_P, _P, _i64, _i64, _i64, _i64, _P, _P]
    L.mp_prescrimp.argtypes = [_P, _P, _i64, _i64, ctypes.c_double, _P, _P, _P]
    L.mp_last_launch_count.argtypes = [_P]
    L.mp_last_near_duplicates.argtypes = [_P]
    L.mp_last_near_duplicates.restype = _i64
    L.mp_last_launch_count.restype = _i64
    L.mp_set_phase_timing.argtypes = [_P, ctypes.c_int]
    L.mp_last_phase_ms.argtypes = [_P, ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double),
                                   ctypes.POINTER(ctypes.c_double)]
    L.mp_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.mp_batch_create.argtypes = [_P, _i64, _P, _P, _P, ctypes.c_int, ctypes.POINTER(_P)]
    L.mp_batch_destroy.argtypes = [_P]
    L.mp_batch_cells.argtypes = [_P]
    L.mp_batch_cells.restype = ctypes.c_double
    L.mp_batch_tiles.argtypes = [_P]
    L.mp_batch_tiles.restype = _i64
    L.mp_batch_launch_count.argtypes = [_P]
    L.mp_batch_launch_count.restype = _i64
    L.mp_batch_upload.argtypes = [_P, _P, _P]
    L.mp_batch_launch.argtypes = [_P, _P]
    L.mp_batch_download.argtypes = [_P, _P, _P, _P]
    L.mp_batch_run.argtypes = [_P, _P, _P, _P, _P]
    L.mp_server_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, _i64,
                                   ctypes.POINTER(_P)]
    L.mp_server_submit.argtypes = [_P, _P, _i64, _i64, ctypes.POINTER(_i64)]
    L.mp_server_poll.argtypes = [_P, _i64, ctypes.POINTER(ctypes.c_int)]
    L.mp_server_collect.argtypes = [_P, _i64, _P, _P, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_double)]
    L.mp_server_stats.argtypes = [_P, ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                  ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                  ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_size_t)]
    L.mp_server_destroy.argtypes = [_P]
    L.mp_list_algorithms.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
    L.mp_run_algorithm.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   _i64, ctypes.c_int]
    _lib = L
    return L


def status_string(status: int) -> str:
    return load_library().mp_status_string(status).decode()


def list_algorithms() -> list[str]:
    L = load_library()
    buf = ctypes.create_string_buffer(4096)
    L.mp_list_algorithms(buf, len(buf))
    return buf.value.decode().split()


def run_algorithm(algo: str, input_file: str, output_file: str, window_length: int,
                  prescrimp_stride: int = 0, blocklen: int = 0, filetype: int = FILETYPE_ASCII,
                  reanchor_k: int = 0, device: int = 0) -> int:
    """One registered variant end to end on files (the reference's main)."""
    L = load_library()
    return L.mp_run_algorithm(algo.encode(), input_file.encode(), output_file.encode(),
                              window_length, prescrimp_stride, blocklen, filetype, reanchor_k,
                              device)


def measure_fma_peak(device: int = 0, which: int = 1) -> float:
    """FLOP/s of the CUDA-core FMA pipe: 0 FP32 FFMA, 1 FP32 f32x2, 2 FP64."""
    v = ctypes.c_double()
    rc = load_library().mp_measure_fma_peak(device, which, ctypes.byref(v))
    if rc != MP_OK:
        raise MpError(rc, status_string(rc))
    return v.value


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return int(a.data_ptr())  # torch tensor (device or host)


@dataclass
class Profile:
    dist2: object   # squared distances (numpy or torch)
    index: object   # neighbour windows

    @property
    def distance(self):
        return np.sqrt(np.abs(np.asarray(self.dist2)))


class Context:
    """One mp_context: a device and its scratch (one per host thread)."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0):
        L = load_library()
        h = _P()
        rc = L.mp_context_create(device, mem_budget_bytes, ctypes.byref(h))
        if rc != MP_OK:
            raise MpError(rc, status_string(rc))
        self._h = h
        self._L = L
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            self._L.mp_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != MP_OK:
            raise MpError(rc, f"{status_string(rc)}: {self._L.mp_last_error(self._h).decode()}")

    def set_phase_timing(self, on: bool = True):
        self._check(self._L.mp_set_phase_timing(self._h, int(on)))

    def last_phase_ms(self) -> tuple[float, float, float]:
        """(preparation, join kernel, finalisation) of the last selfjoin, in ms."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self._L.mp_last_phase_ms(self._h, ctypes.byref(a), ctypes.byref(b),
                                             ctypes.byref(c)))
        return a.value, b.value, c.value

    @property
    def last_launch_count(self) -> int:
        return int(self._L.mp_last_launch_count(self._h))

    @property
    def last_near_duplicates(self) -> int:
        """Guarded form: windows the last self-join recomputed pairwise in FP64."""
        return int(self._L.mp_last_near_duplicates(self._h))

    def selfjoin(self, A, m: int, precision: int = FP64, reanchor_k: int = 0,
                 blocklen: int = 0, diag_lo: int = 0, diag_hi: int = 0, excl: int = -1,
                 out=None, stream=None) -> Profile:
        """Self-join of series A (numpy float64 on the host, or a CUDA tensor).

        Returns squared distances and neighbour indices for every window, in the
        memory space of ``out`` (numpy arrays by default)."""
        if isinstance(A, np.ndarray):
            A = np.ascontiguousarray(A, dtype=np.float64)
            n = A.size
        else:
            n = A.numel()
        PL = n - m + 1
        if out is None:
            d2 = np.empty(max(PL, 0), dtype=np.float64)
            ix = np.empty(max(PL, 0), dtype=np.int64)
        else:
            d2, ix = out
        rc = self._L.mp_selfjoin(self._h, _ptr(A), n, m, excl, precision, reanchor_k, blocklen,
                                 diag_lo, diag_hi, _ptr(d2), _ptr(ix), stream)
        self._check(rc)
        return Profile(d2, ix)

    def selfjoin_ranges(self, A, m: int, ranges, precision: int = FP64, reanchor_k: int = 0,
                        blocklen: int = 0, excl: int = -1, out=None, stream=None) -> Profile:
        """selfjoin over several diagonal ranges [(lo, hi), ...] in one call (one
        preparation and one synchronisation): a rank's part of a sharded join."""
        if isinstance(A, np.ndarray):
            A = np.ascontiguousarray(A, dtype=np.float64)
            n = A.size
        else:
            n = A.numel()
        PL = n - m + 1
        if out is None:
            d2 = np.empty(max(PL, 0), dtype=np.float64)
            ix = np.empty(max(PL, 0), dtype=np.int64)
        else:
            d2, ix = out
        flat = np.ascontiguousarray(np.asarray(ranges, dtype=np.int64).reshape(-1))
        rc = self._L.mp_selfjoin_ranges(self._h, _ptr(A), n, m, excl, precision, reanchor_k,
                                        blocklen, flat.ctypes.data if flat.size else None,
                                        flat.size // 2, _ptr(d2), _ptr(ix), stream)
        self._check(rc)
        return Profile(d2, ix)

    def prescrimp(self, A, m: int, stride: float, out=None, stream=None) -> Profile:
        """PreSCRIMP approximate profile (the SCRIMP++ front end): query windows
        every floor(stride * m), their whole distance profiles and the walks along
        each query's best diagonal.  Squared distances; +inf / index 0 where no
        evaluated cell reached a window."""
        if isinstance(A, np.ndarray):
            A = np.ascontiguousarray(A, dtype=np.float64)
            n = A.size
        else:
            n = A.numel()
        PL = n - m + 1
        if out is None:
            d2 = np.empty(max(PL, 0), dtype=np.float64)
            ix = np.empty(max(PL, 0), dtype=np.int64)
        else:
            d2, ix = out
        self._check(self._L.mp_prescrimp(self._h, _ptr(A), n, m, float(stride), _ptr(d2),
                                         _ptr(ix), stream))
        return Profile(d2, ix)

    def window_stats(self, A, m: int):
        A = np.ascontiguousarray(A, dtype=np.float64)
        PL = A.size - m + 1
        muS = np.empty(PL)
        sInv = np.empty(PL)
        self._check(self._L.mp_window_stats(self._h, _ptr(A), A.size, m, _ptr(muS), _ptr(sInv),
                                            None))
        return muS, sInv

    def first_qt(self, A, m: int, d_lo: int, d_hi: int):
        A = np.ascontiguousarray(A, dtype=np.float64)
        qt = np.empty(max(d_hi - d_lo, 0))
        self._check(self._L.mp_first_qt(self._h, _ptr(A), A.size, m, d_lo, d_hi, _ptr(qt),
                                        None))
        return qt

    def eval_diag_block_triangle(self, prof_colmin, idx_colmin, prof_rowmin, idx_rowmin, tmpQ,
                                 blocklen, trianglen, A_hor, A_vert, m, s_hor, mu_hor, s_vert,
                                 mu_vert, baserow, basecol):
        """The reference kernel's contract; numpy views are updated in place."""
        self._check(self._L.mp_eval_diag_block_triangle(
            self._h, _ptr(prof_colmin), _ptr(idx_colmin), _ptr(prof_rowmin), _ptr(idx_rowmin),
            _ptr(tmpQ), blocklen, trianglen, _ptr(A_hor), _ptr(A_vert), m, _ptr(s_hor),
            _ptr(mu_hor), _ptr(s_vert), _ptr(mu_vert), baserow, basecol, None))


class Batch:
    """Many self-joins in one persistent, graph-captured launch (FP32 form).

    ``lengths``/``windows`` fix the plan; ``reanchor_k`` is one interval per
    series (None: the autotuned table, see thesiscode_b200.autotune).  Input
    series are float32 (``input_f32=True``) or float64 numpy arrays."""

    def __init__(self, ctx: Context, lengths, windows, reanchor_k=None, input_f32: bool = True):
        self._L = ctx._L
        self._ctx = ctx
        self.lengths = np.ascontiguousarray(lengths, dtype=np.int64)
        self.windows = np.ascontiguousarray(windows, dtype=np.int64)
        if reanchor_k is None:
            from thesiscode_b200 import autotune
            reanchor_k = [autotune.lookup(int(n), int(m)) for n, m in zip(self.lengths,
                                                                          self.windows)]
        self.reanchor_k = np.ascontiguousarray(reanchor_k, dtype=np.int64)
        self.input_f32 = input_f32
        h = _P()
        rc = self._L.mp_batch_create(ctx._h, self.lengths.size, self.lengths.ctypes.data,
                                     self.windows.ctypes.data, self.reanchor_k.ctypes.data,
                                     1 if input_f32 else 0, ctypes.byref(h))
        if rc != MP_OK:
            raise MpError(rc, status_string(rc))
        self._h = h
        self._keep = []

    @property
    def cells(self) -> float:
        return float(self._L.mp_batch_cells(self._h))

    @property
    def tiles(self) -> int:
        return int(self._L.mp_batch_tiles(self._h))

    @property
    def launch_count(self) -> int:
        return int(self._L.mp_batch_launch_count(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._L.mp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != MP_OK:
            raise MpError(rc, status_string(rc))

    def upload(self, series, stream=None):
        dt = np.float32 if self.input_f32 else np.float64
        arrs = [np.ascontiguousarray(x, dtype=dt) for x in series]
        if len(arrs) != self.lengths.size or any(a.size != n for a, n in zip(arrs, self.lengths)):
            raise ValueError("series do not match the plan")
        ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        self._check(self._L.mp_batch_upload(self._h, ptrs, stream))
        self._keep = arrs

    def launch(self, stream=None):
        self._check(self._L.mp_batch_launch(self._h, stream))

    def outputs(self) -> list[Profile]:
        """Output arrays for every series of the plan, to reuse across runs (fresh
        arrays pay page faults on every download)."""
        pls = self.lengths - self.windows + 1
        return [Profile(np.empty(int(p)), np.empty(int(p), dtype=np.int64)) for p in pls]

    def download(self, stream=None, out=None) -> list[Profile]:
        """Copies the profiles to the host, into ``out`` (from outputs()) when given."""
        if out is None:
            out = self.outputs()
        d2 = [p.dist2 for p in out]
        ix = [p.index for p in out]
        dp = (ctypes.c_void_p * len(d2))(*[a.ctypes.data for a in d2])
        ip = (ctypes.c_void_p * len(ix))(*[a.ctypes.data for a in ix])
        self._check(self._L.mp_batch_download(self._h, dp, ip, stream))
        return [Profile(a, b) for a, b in zip(d2, ix)]

    def run(self, series, stream=None, out=None) -> list[Profile]:
        self.upload(series, stream)
        self.launch(stream)
        return self.download(stream, out)


class Server:
    """Continuous-batching request server (mp_server_*): submit self-joins,
    collect profiles; admission by device-memory budget, at most `slots`
    requests admitted at once.  The FP32 re-anchored form runs the admitted
    requests together as epochs of the persistent tile kernel; the FP64 and
    guarded forms run `slots` workers, each on its own stream."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 8 << 30, slots: int = 4,
                 precision: int = FP32_REANCHOR, reanchor_k: int = 1024):
        self._L = load_library()
        h = _P()
        rc = self._L.mp_server_create(device, mem_budget_bytes, slots, precision, reanchor_k,
                                      ctypes.byref(h))
        if rc != MP_OK:
            raise MpError(rc, status_string(rc))
        self._h = h
        self._pl = {}

    def submit(self, A, m: int) -> tuple[int, int]:
        """Returns (ticket, status); status MP_ERR_BUDGET means rejected."""
        A = np.ascontiguousarray(A, dtype=np.float64)
        t = _i64()
        rc = self._L.mp_server_submit(self._h, A.ctypes.data, A.size, m, ctypes.byref(t))
        if rc not in (MP_OK, MP_ERR_BUDGET):
            raise MpError(rc, status_string(rc))
        self._pl[t.value] = A.size - m + 1
        return t.value, rc

    def done(self, ticket: int) -> bool:
        st = ctypes.c_int()
        return self._L.mp_server_poll(self._h, ticket, ctypes.byref(st)) == 1

    def collect(self, ticket: int, want_profile: bool = True):
        """Waits; returns (status, Profile or None, latency_s, queue_s)."""
        PL = self._pl.pop(ticket)
        d2 = np.empty(PL) if want_profile else None
        ix = np.empty(PL, dtype=np.int64) if want_profile else None
        lat, que = ctypes.c_double(), ctypes.c_double()
        rc = self._L.mp_server_collect(self._h, ticket, _ptr(d2), _ptr(ix), ctypes.byref(lat),
                                       ctypes.byref(que))
        prof = Profile(d2, ix) if (want_profile and rc == MP_OK) else None
        return rc, prof, lat.value, que.value

    def stats(self) -> dict:
        c, r, w, u = _i64(), _i64(), _i64(), _i64()
        cells = ctypes.c_double()
        used = ctypes.c_size_t()
        self._L.mp_server_stats(self._h, ctypes.byref(c), ctypes.byref(r), ctypes.byref(w),
                                ctypes.byref(u), ctypes.byref(cells), ctypes.byref(used))
        return {"completed": c.value, "rejected": r.value, "waiting": w.value,
                "running": u.value, "cells": cells.value, "bytes_in_use": used.value}

    def close(self):
        if getattr(self, "_h", None):
            self._L.mp_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cells(n: int, m: int, diag_lo: int = 0, diag_hi: int = 0, excl: int = -1) -> int:
    """Distance-matrix cells a self-join evaluates on diagonals [diag_lo, diag_hi)."""
    PL = n - m + 1
    excl = m // 4 if excl < 0 else excl
    if diag_lo == 0 and diag_hi == 0:
        diag_lo, diag_hi = excl + 1, PL
    diag_lo = max(diag_lo, excl + 1)
    diag_hi = min(diag_hi, PL)
    if diag_hi <= diag_lo:
        return 0
    a, b = PL - diag_lo, PL - diag_hi + 1  # lengths of first and last diagonal
    return (a + b) * (diag_hi - diag_lo) // 2
