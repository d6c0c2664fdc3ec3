"""CPU restatement of PreSCRIMP -- TEST INFRASTRUCTURE (the checker for
mp_prescrimp; never part of the product path).

Pinned against the reference's own PreSCRIMP (scrimppp/src/ScrimpppOrig.cpp:
130-266), built unchanged as oracle/_ref/scrimppp_ref_orig.  That code
convolves with FFTW, which is not installed here; oracle/ref_fftw_stub.cpp
stands in for the FFTW calls it makes.  tests/golden/prescrimp_ref.npz holds
its outputs (tests/golden/make_prescrimp_golden.py) and
tests/test_prescrimp_oracle.py holds this restatement to them: distances
within 1e-9 relative (1e-6 at a 1e4 level offset, where the FFT's own rounding
dominates), indices equal.  Differences from the reference, shared with the GPU
implementation: query rows are direct FP64 dot products (not FFT
convolutions), and every update is a min-merge, so the result does not depend
on the shuffled query order (the reference assigns a query's row minimum to
its own entry, :209-210, which differs from a min-merge only by rounding).  A
flat query window (zero variance) leaves the reference's row minimum index
uninitialised (:196-211); the restatement skips such a query's walk.
"""
from __future__ import annotations

import math

import numpy as np


def orig_stats(x: np.ndarray, m: int):
    """Means and standard deviations, ScrimpppOrig.cpp:86-107 (prefix sums in
    index order, variance = S2/m - mean^2)."""
    n = x.size
    cs = np.add.accumulate(x)
    cs2 = np.add.accumulate(x * x)
    s = np.empty(n - m + 1)
    s2 = np.empty(n - m + 1)
    s[0], s2[0] = cs[m - 1], cs2[m - 1]
    s[1:] = cs[m:] - cs[:n - m]
    s2[1:] = cs2[m:] - cs2[:n - m]
    mean = s / m
    sigma = np.sqrt(s2 / m - mean * mean)
    return mean, sigma


def _distance(m, qt, mean_j, mean_i, sig_j, sig_i):
    # ScrimpppOrig.cpp:195: 2 * (m - (qt - m * mean_j * mean_i) / (sigma_j * sigma_i))
    return 2.0 * (m - (qt - m * mean_j * mean_i) / (sig_j * sig_i))


def prescrimp(x, m: int, stride: float):
    """(squared distances, indices) after PreSCRIMP; +inf / 0 where no
    evaluated cell reached a window."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.size
    PL = n - m + 1
    excl = m // 4                                   # :73
    step = int(math.floor(stride * m))              # :49
    mean, sigma = orig_stats(x, m)
    W = np.lib.stride_tricks.sliding_window_view(x, m)
    prof = np.full(PL, np.inf)
    idx = np.zeros(PL, dtype=np.int64)
    fm = float(m)

    def lower(w, d, nb):
        if d < prof[w]:
            prof[w] = d
            idx[w] = nb

    with np.errstate(divide="ignore", invalid="ignore"):
        for i in range(0, PL, step):                # :155-157 (order irrelevant here)
            qt = W @ x[i:i + m]
            d = _distance(fm, qt, mean, mean[i], sigma, sigma[i])
            d[max(i - excl + 1, 0):min(i + excl, PL)] = np.inf   # :190-193
            upd = d < prof                          # :203-207
            prof[upd] = d[upd]
            idx[upd] = i
            j = int(np.argmin(np.where(np.isnan(d), np.inf, d)))   # :198-201, first minimum
            dmin = float(d[j])
            if not dmin < np.inf:
                continue
            lower(i, dmin, j)
            z0 = (fm - dmin / 2.0) * (sigma[j] * sigma[i]) + fm * mean[j] * mean[i]   # :213
            z = z0
            k = 1
            while k < step and i + k < PL and j + k < PL:                              # :216-229
                z = z - x[i + k - 1] * x[j + k - 1] + x[i + k + m - 1] * x[j + k + m - 1]
                dd = _distance(fm, z, mean[j + k], mean[i + k], sigma[j + k], sigma[i + k])
                lower(i + k, dd, j + k)
                lower(j + k, dd, i + k)
                k += 1
            z = z0
            k = 1
            while k < step and i - k >= 0 and j - k >= 0:                              # :231-244
                z = z - x[i - k + m] * x[j - k + m] + x[i - k] * x[j - k]
                dd = _distance(fm, z, mean[j - k], mean[i - k], sigma[j - k], sigma[i - k])
                lower(i - k, dd, j - k)
                lower(j - k, dd, i - k)
                k += 1
    return prof, idx
