// Per-window preparation kernels: window statistics, first dot products and
// the packed row/column records the join kernels stream.
//
// Two statistics paths:
//  * reference-exact (FP64 form): the reference's prefix-sum formula,
//    scrimppp/src/ScrimpSequOpt.cpp:33-79, evaluated with explicitly rounded
//    operations (__dadd_rn/__dmul_rn/... are never contracted into FMAs) so the
//    result is bit-identical to the reference built with IEEE semantics.  The
//    prefix sums are a dependent chain and run on one thread.
//  * FP64 Welford (FP32 form): each thread slides Welford's mean/M2 update
//    over a chunk of windows, restarting from a fresh Welford pass at every
//    chunk start; exact zero-variance windows are found with an integer count
//    of value changes, so a constant window at any level is flagged exactly.
#include "mp_common.cuh"
#include "mp_kernels.h"
#include "mp_prep_device.cuh"

namespace mpgpu {

// ---- reference-exact statistics -------------------------------------------

// cs[i] = A[i] + cs[i-1], cs2[i] = A[i]*A[i] + cs2[i-1] in index order
// (ScrimpSequOpt.cpp:43-49).  Each chain is inherently serial, so lane 0 of
// warp 0 runs the sum of A and lane 1 the sum of A*A, side by side, out of
// shared memory: the block's other warps load the next chunk of A and write
// the previous chunk's sums back (both coalesced) meanwhile, so neither chain
// waits for global memory.  Launch with kPrefixThreads threads in one block.
__global__ void __launch_bounds__(kPrefixThreads)
    ref_prefix_kernel(const double* __restrict__ A, int64_t n, double* __restrict__ cs,
                      double* __restrict__ cs2) {
    constexpr int C = kPrefixChunk;
    __shared__ double in[2][C];
    __shared__ double out[2][2][C];  // [chain][buffer][k]: chain 0 sums A, chain 1 sums A*A
    if (blockIdx.x != 0) return;
    const int t = threadIdx.x;
    const int64_t nch = (n + C - 1) / C;
    for (int k = t; k < C; k += blockDim.x) in[0][k] = k < n ? A[k] : 0.0;
    __syncthreads();
    double acc = 0.0;
    for (int64_t c = 0; c < nch; ++c) {
        const int b = (int)(c & 1);
        if (t < 2) {
            const int64_t base = c * C;
            const int cnt = (int)min((int64_t)C, n - base);
            const double* src = in[b];
            double* dst = out[t][b];
            int k = 0;
            if (base == 0) {
                acc = t == 0 ? src[0] : __dmul_rn(src[0], src[0]);
                dst[0] = acc;
                k = 1;
            }
            for (; k + 8 <= cnt; k += 8) {
                double a[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) a[i] = src[k + i];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    acc = __dadd_rn(t == 0 ? a[i] : __dmul_rn(a[i], a[i]), acc);
                    dst[k + i] = acc;
                }
            }
            for (; k < cnt; ++k) {
                const double a = src[k];
                acc = __dadd_rn(t == 0 ? a : __dmul_rn(a, a), acc);
                dst[k] = acc;
            }
        } else if (t >= 32) {
            const int tt = t - 32, nt = blockDim.x - 32;
            if (c + 1 < nch)
                for (int k = tt; k < C; k += nt) {
                    const int64_t i = (c + 1) * C + k;
                    in[b ^ 1][k] = i < n ? A[i] : 0.0;
                }
            if (c >= 1)
                for (int k = tt; k < C; k += nt) {
                    const int64_t i = (c - 1) * C + k;
                    cs[i] = out[0][b ^ 1][k];
                    cs2[i] = out[1][b ^ 1][k];
                }
        }
        __syncthreads();
    }
    const int64_t c = nch - 1;
    for (int k = t; k < C; k += blockDim.x) {
        const int64_t i = c * C + k;
        if (i < n) {
            cs[i] = out[0][c & 1][k];
            cs2[i] = out[1][c & 1][k];
        }
    }
}

// Window sums from prefix differences, mean = S/m, var = S2/m - mean^2,
// sInv = 1/sqrt(var), muS = (mean*sInv)*sqrt(m) (ScrimpSequOpt.cpp:50-68).
__global__ void ref_stats_kernel(const double* __restrict__ cs, const double* __restrict__ cs2,
                                 int64_t PL, int64_t m, double* __restrict__ muS,
                                 double* __restrict__ sInv) {
    const double dm = (double)m;
    const double sqrt_m = __dsqrt_rn(dm);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < PL;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double s = (i == 0) ? cs[m - 1] : __dsub_rn(cs[m - 1 + i], cs[i - 1]);
        const double s2 = (i == 0) ? cs2[m - 1] : __dsub_rn(cs2[m - 1 + i], cs2[i - 1]);
        const double mean = __ddiv_rn(s, dm);
        const double var = __dsub_rn(__ddiv_rn(s2, dm), __dmul_rn(mean, mean));
        const double si = __ddiv_rn(1.0, __dsqrt_rn(var));
        sInv[i] = si;
        muS[i] = __dmul_rn(__dmul_rn(mean, si), sqrt_m);
    }
}

// First dot product per diagonal, summed in k order without fusion
// (ScrimpSequOpt.cpp:81-96).  Consecutive threads take consecutive diagonals
// so the A[k+d] reads coalesce and A[k] is a broadcast.
__global__ void first_qt_kernel(const double* __restrict__ A, int64_t m, int64_t d_lo,
                                int64_t d_hi, double* __restrict__ qt) {
    for (int64_t d = d_lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; d < d_hi;
         d += (int64_t)gridDim.x * blockDim.x) {
        double z = 0.0;
        const double* a = A + d;
        for (int64_t k = 0; k < m; ++k) z = __dadd_rn(z, __dmul_rn(__ldg(a + k), __ldg(A + k)));
        qt[d - d_lo] = z;
    }
}

// Row/column record of the FP64 join: {A[i], A[i+m], sInv[i], muS[i]}.
// `Apad` holds n+1 values (A[n] = 0 feeds only the update after a diagonal's
// last cell, whose result is never used).
__global__ void pack_fp64_kernel(const double* __restrict__ Apad, int64_t m, int64_t count,
                                 const double* __restrict__ sInv, const double* __restrict__ muS,
                                 double4* __restrict__ rec) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        rec[i] = make_double4(Apad[i], Apad[i + m], sInv[i], muS[i]);
    }
}

// ---- FP64 Welford statistics (FP32 form) ----------------------------------

// chg[i] = 1 if A[i] != A[i-1] (i >= 1), chg[0] = 0; an inclusive scan of chg
// gives the number of value changes up to i.
__global__ void change_flags_kernel(const double* __restrict__ A, int64_t n, int* __restrict__ chg) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        chg[i] = (i > 0 && A[i] != A[i - 1]) ? 1 : 0;
}

// Block-level inclusive scan helper (Hillis-Steele over a warp, then warps).
__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(kFullMask, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Two-level inclusive scan of int flags: per-block scan + block totals.
__global__ void scan_blocks_kernel(int* __restrict__ x, int64_t n, int* __restrict__ block_tot) {
    __shared__ int wsum[32];
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int v = (i < n) ? x[i] : 0;
    v = warp_incl_scan(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 31) wsum[w] = v;
    __syncthreads();
    if (w == 0) {
        int t = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
        t = warp_incl_scan(t);
        wsum[lane] = t;
    }
    __syncthreads();
    if (w > 0) v += wsum[w - 1];
    if (i < n) x[i] = v;
    if (threadIdx.x == blockDim.x - 1) block_tot[blockIdx.x] = v;
}

__global__ void scan_totals_kernel(int* __restrict__ tot, int64_t nblocks) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int s = 0;
    for (int64_t b = 0; b < nblocks; ++b) {
        s += tot[b];
        tot[b] = s;
    }
}

__global__ void scan_add_kernel(int* __restrict__ x, int64_t n, const int* __restrict__ tot) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n && blockIdx.x > 0) x[i] += tot[blockIdx.x - 1];
}

// Welford statistics per chunk of windows (see welford_chunk).
__global__ void welford_kernel(const double* __restrict__ A, int64_t m, int64_t PL, int64_t chunk,
                               const int* __restrict__ nchg, double* __restrict__ mean_out,
                               double* __restrict__ norm_out) {
    const int64_t nthreads = (PL + chunk - 1) / chunk;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nthreads;
         t += (int64_t)gridDim.x * blockDim.x)
        welford_chunk(A, m, PL, chunk, t, nchg, mean_out, norm_out);
}

// Row and column records of the FP32 form (see pack_fp32_record).
__global__ void pack_fp32_kernel(const double* __restrict__ A, int64_t m, int64_t PL, int H,
                                 int64_t count, const double* __restrict__ mean,
                                 const double* __restrict__ norm, float4* __restrict__ rowrec,
                                 float4* __restrict__ colrec) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < count;
         j += (int64_t)gridDim.x * blockDim.x)
        pack_fp32_record(A, m, PL, H, mean, norm, j, rowrec, colrec);
}

}  // namespace mpgpu
