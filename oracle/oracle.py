"""CPU oracle bindings -- TEST INFRASTRUCTURE.

ctypes front end for
  * ``libscrimp_oracle.so``: the plain-C restatement of the reference's
    diagonal-blocked SCRIMP hot path (oracle/scrimp_oracle.c), and
  * ``_ref/libscrimp_ref_{ieee,fast}.so``: the reference's own sources
    compiled unchanged (oracle/Makefile), present where the reference tree was
    available at build time.

The same recipe builds command-line programs of the reference, run as
subprocesses by the tests and the golden-fixture scripts: ``scrimppp_ref_ieee``
and ``scrimppp_ref_fast`` (its CLI), ``scrimppp_ref_orig`` (plus SCRIMP++ over
a stand-in FFT) and ``scrimppp_ref_bin`` (plus its binary MPI-IO file classes
over a single-rank emulation).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only to check or time the reference algorithm on the host.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference's scrimppp directory (sources, data_testing/).  Needed only to
# build oracle/_ref or to regenerate the golden fixtures; unset means absent.
REF_SRC = os.environ.get("SCRIMP_REF_ROOT", "")

_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_int64)
_i64 = ctypes.c_int64


def build(with_reference: bool | None = None) -> None:
    """Compile the C restatement, and the reference-source oracle when the
    reference tree is present (or ``with_reference`` forces it)."""
    targets = ["oracle"]
    if with_reference and not REF_SRC:
        raise RuntimeError("oracle.build(with_reference=True) needs SCRIMP_REF_ROOT: the "
                           "reference's scrimppp directory")
    if with_reference or (with_reference is None and REF_SRC and os.path.isdir(REF_SRC)):
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REF_SRC}", *targets], check=True)


def _dptr(a):
    return a.ctypes.data_as(_D)


def _lptr(a):
    return a.ctypes.data_as(_L)


class Oracle:
    """The C restatement (always available once built)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "libscrimp_oracle.so")
        if not os.path.exists(path):
            build(with_reference=False)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.orc_window_stats.argtypes = [_D, _i64, _i64, _D, _D]
        L.orc_first_qt.argtypes = [_D, _i64, _i64, _i64, _i64, _D]
        L.orc_eval_diag_block_triangle.argtypes = [_D, _L, _D, _L, _D, _i64, _i64, _D, _D, _i64,
                                                   _D, _D, _D, _D, _i64, _i64]
        L.orc_selfjoin_fp64.argtypes = [_D, _i64, _i64, _i64, _i64, _i64, _i64, ctypes.c_int,
                                        _D, _L]
        L.orc_pair_d2.argtypes = [_D, _i64, _i64, _i64, _i64]
        L.orc_cell_scores.argtypes = [_D, _i64, _i64, _i64, _i64, _D, _D, _i64, _L, _L, _D]
        L.orc_pair_d2.restype = ctypes.c_double
        L.orc_cells.argtypes = [_i64, _i64, _i64, _i64]
        L.orc_cells.restype = ctypes.c_double

    def window_stats(self, A, m):
        A = np.ascontiguousarray(A, dtype=np.float64)
        PL = A.size - m + 1
        muS = np.empty(PL)
        sInv = np.empty(PL)
        rc = self.lib.orc_window_stats(_dptr(A), A.size, m, _dptr(muS), _dptr(sInv))
        assert rc == 0, rc
        return muS, sInv

    def first_qt(self, A, m, d_lo, d_hi):
        A = np.ascontiguousarray(A, dtype=np.float64)
        out = np.empty(max(d_hi - d_lo, 0))
        rc = self.lib.orc_first_qt(_dptr(A), A.size, m, d_lo, d_hi, _dptr(out))
        assert rc == 0, rc
        return out

    def selfjoin(self, A, m, blocklen=500, diag_lo=0, diag_hi=0, excl=-1, nthreads=None):
        """Returns (d2[PL], idx[PL]) like ScrimpVertBlocked (index init 0)."""
        A = np.ascontiguousarray(A, dtype=np.float64)
        PL = A.size - m + 1
        d2 = np.empty(PL)
        idx = np.empty(PL, dtype=np.int64)
        nthreads = nthreads or min(os.cpu_count() or 1, 16)
        rc = self.lib.orc_selfjoin_fp64(_dptr(A), A.size, m, excl, blocklen, diag_lo, diag_hi,
                                        nthreads, _dptr(d2), _lptr(idx))
        assert rc == 0, rc
        return d2, idx

    def eval_diag_block_triangle(self, prof_col, idx_col, prof_row, idx_row, tmpQ, blocklen,
                                 trianglen, A_hor, A_vert, m, s_hor, mu_hor, s_vert, mu_vert,
                                 baserow, basecol):
        """Array views are mutated in place, as in the reference."""
        self.lib.orc_eval_diag_block_triangle(_dptr(prof_col), _lptr(idx_col), _dptr(prof_row),
                                              _lptr(idx_row), _dptr(tmpQ), blocklen, trianglen,
                                              _dptr(A_hor), _dptr(A_vert), m, _dptr(s_hor),
                                              _dptr(mu_hor), _dptr(s_vert), _dptr(mu_vert),
                                              baserow, basecol)

    def cell_scores(self, A, m, cols, rows, blocklen=500, excl=-1, stats=None):
        """Scores the reference's arithmetic gives cells (cols[k], rows[k]) in a
        vert_blocked join with this blocklen (cols[k] < rows[k])."""
        A = np.ascontiguousarray(A, dtype=np.float64)
        muS, sInv = stats if stats is not None else self.window_stats(A, m)
        c = np.ascontiguousarray(cols, dtype=np.int64)
        r = np.ascontiguousarray(rows, dtype=np.int64)
        out = np.empty(c.size)
        rc = self.lib.orc_cell_scores(_dptr(A), A.size, m, excl, blocklen, _dptr(muS),
                                      _dptr(sInv), c.size, _lptr(c), _lptr(r), _dptr(out))
        assert rc == 0, rc
        return out

    def pair_d2(self, A, m, i, j):
        A = np.ascontiguousarray(A, dtype=np.float64)
        return self.lib.orc_pair_d2(_dptr(A), A.size, m, int(i), int(j))

    def cells(self, n, m, diag_lo, diag_hi):
        return self.lib.orc_cells(n, m, diag_lo, diag_hi)


class RefOracle:
    """The reference's own sources (oracle/_ref); ``flavour`` is 'ieee' or 'fast'."""

    def __init__(self, flavour: str = "ieee"):
        path = os.path.join(REF_DIR, f"libscrimp_ref_{flavour}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.flavour = flavour
        L = self.lib
        L.ref_window_stats.argtypes = [_D, _i64, _i64, _D, _D]
        L.ref_first_qt.argtypes = [_D, _i64, _i64, _i64, _i64, _D]
        L.ref_eval_diag_block_triangle.argtypes = [_D, _L, _D, _L, _D, _i64, _i64, _D, _D, _i64,
                                                   _D, _D, _D, _D, _i64, _i64]
        L.ref_vert_blocked.argtypes = [_D, _i64, _i64, _i64, ctypes.c_int, _D, _L, _D]
        L.ref_triv_par_threads.argtypes = [_D, _i64, _i64, _i64, _i64, _i64, ctypes.c_int, _D,
                                           _L, _D]

    @staticmethod
    def available(flavour: str = "ieee") -> bool:
        return os.path.exists(os.path.join(REF_DIR, f"libscrimp_ref_{flavour}.so"))

    def window_stats(self, A, m):
        A = np.ascontiguousarray(A, dtype=np.float64)
        PL = A.size - m + 1
        muS = np.empty(PL)
        sInv = np.empty(PL)
        assert self.lib.ref_window_stats(_dptr(A), A.size, m, _dptr(muS), _dptr(sInv)) == 0
        return muS, sInv

    def first_qt(self, A, m, first, last_inclusive):
        A = np.ascontiguousarray(A, dtype=np.float64)
        out = np.empty(last_inclusive - first + 1)
        assert self.lib.ref_first_qt(_dptr(A), A.size, m, first, last_inclusive, _dptr(out)) == 0
        return out

    def vert_blocked(self, A, m, blocklen=500, shuffle=True):
        A = np.ascontiguousarray(A, dtype=np.float64)
        PL = A.size - m + 1
        d2 = np.empty(PL)
        idx = np.empty(PL, dtype=np.int64)
        sec = ctypes.c_double(0)
        rc = self.lib.ref_vert_blocked(_dptr(A), A.size, m, blocklen, int(shuffle), _dptr(d2),
                                       _lptr(idx), ctypes.byref(sec))
        assert rc == 0, rc
        return d2, idx, sec.value

    def triv_par_threads(self, A, m, diag_lo, diag_hi, nthreads, blocklen=500):
        A = np.ascontiguousarray(A, dtype=np.float64)
        PL = A.size - m + 1
        d2 = np.empty(PL)
        idx = np.empty(PL, dtype=np.int64)
        sec = ctypes.c_double(0)
        rc = self.lib.ref_triv_par_threads(_dptr(A), A.size, m, blocklen, diag_lo, diag_hi,
                                           nthreads, _dptr(d2), _lptr(idx), ctypes.byref(sec))
        assert rc == 0, rc
        return d2, idx, sec.value

    def eval_diag_block_triangle(self, *args):
        conv = []
        for a in args:
            if isinstance(a, np.ndarray):
                conv.append(_lptr(a) if a.dtype == np.int64 else _dptr(a))
            else:
                conv.append(a)
        self.lib.ref_eval_diag_block_triangle(*conv)
