// Guarded FP32 form: FP64 tiles where the data is ill-conditioned for an FP32
// running sum.
//
// The FP32 recurrence's rounding error is relative to the covariance it
// carries, so a diagonal that passes, within one re-anchor interval, from
// windows of large norm (a level step on a walk, values straddling a constant
// stretch) to windows of far smaller norm carries a large absolute error into
// the small cells.  A window is a hazard when its norm is more than
// kGuardRatio times smaller than the largest norm among the K + 32R windows
// before it (that span covers every cell a tile can carry into it), or when it
// is flat.  Tiles whose column or row windows include a hazard are left out of
// the FP32 kernel and evaluated here with the same centred recurrence in FP64;
// both kernels min-merge into the same (ordered u, neighbour) keys.  On a
// plain random walk no window is a hazard.
#include <algorithm>
#include <cfloat>

#include "mp_common.cuh"
#include "mp_kernels.h"

namespace mpgpu {

namespace {

constexpr unsigned long long kNoKey = ~0ull;

__device__ __forceinline__ unsigned long long guard_key(float u, int64_t nb) {
    return ((unsigned long long)ord_f32(u) << 32) | (unsigned long long)nb;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(kFullMask, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// One band's tile (columns [j0, j1) of 32R diagonals) in FP64: lane l owns
// diagonals g0 + a, a < R.  Row keys of a chunk of R columns live in 2R - 1
// register slots (slot b + a holds row jc + g0 + b + a); the lower R are
// complete after the chunk and go to global memory with atomicMin.
template <int R>
__device__ void tile_guard(const Fp32TileParams& P, int64_t band, int64_t seg, int lane) {
    const int64_t gb = P.g_lo + band * (int64_t)(32 * R);
    const int64_t g0 = gb + (int64_t)lane * R;
    const int64_t jmax = P.PL - gb;
    const int64_t j0 = seg * P.K;
    const int64_t j1 = min(j0 + P.K, jmax);
    if (j0 >= j1 || !fp32_tile_hazardous(P, gb, j0, j1, 32 * R)) return;
    const float ulim = (float)(1.0 + 1.0 / (double)P.m);
    const double mm = (double)P.m;

    double nc[R];  // m mean_j mean_r - sum A[j+k] A[r+k]  (= -covariance)
#pragma unroll
    for (int a = 0; a < R; ++a) {
        const int64_t g = g0 + a;
        nc[a] = 0.0;
        if (g < P.g_hi && j0 + g < P.PL) {
            double q = 0.0;
            for (int64_t k = 0; k < P.m; ++k) q = __fma_rn(P.A[j0 + k], P.A[j0 + g + k], q);
            nc[a] = __fma_rn(mm * P.mean[j0], P.mean[j0 + g], -q);
        }
    }
    unsigned long long rk[2 * R];
#pragma unroll
    for (int s = 0; s < 2 * R; ++s) rk[s] = kNoKey;

    int64_t jc = j0;
    for (; jc < j1; jc += R) {
#pragma unroll
        for (int b = 0; b < R; ++b) {
            const int64_t j = jc + b;
            const bool vj = j < j1;
            const double dfj = vj ? P.df[j] : 0.0, dgj = vj ? P.dg[j] : 0.0;
            const double nnj = vj ? P.norm[j] : 0.0;
            unsigned long long ck = kNoKey;
#pragma unroll
            for (int a = 0; a < R; ++a) {
                const int64_t g = g0 + a;
                const int64_t r = j + g;
                if (vj && g < P.g_hi && r < P.PL) {
                    const double u = __fma_rn(nc[a], nnj * P.norm[r], 1.0);
                    const float fu = (float)u;
                    if (fu < ulim) {  // NaN (a flat window) never passes
                        const unsigned long long kc = guard_key(fu, r);
                        const unsigned long long kr = guard_key(fu, j);
                        ck = kc < ck ? kc : ck;
                        rk[b + a] = kr < rk[b + a] ? kr : rk[b + a];
                    }
                    nc[a] = __fma_rn(-dfj, P.dg[r], nc[a]);
                    nc[a] = __fma_rn(P.df[r], -dgj, nc[a]);
                }
            }
            ck = warp_min_u64(ck);
            if (lane == 0 && ck != kNoKey) atomicMin(P.key + j, ck);
        }
#pragma unroll
        for (int s = 0; s < R; ++s)
            if (rk[s] != kNoKey) atomicMin(P.key + (jc + g0 + s), rk[s]);
#pragma unroll
        for (int s = 0; s < R - 1; ++s) rk[s] = rk[s + R];
#pragma unroll
        for (int s = R - 1; s < 2 * R; ++s) rk[s] = kNoKey;
    }
#pragma unroll
    for (int s = 0; s < R - 1; ++s)
        if (rk[s] != kNoKey) atomicMin(P.key + (jc + g0 + s), rk[s]);
}

// Same tile space and order as fp32_join_kernel; only hazard tiles do work.
template <int R>
__global__ void __launch_bounds__(128) fp64_guard_kernel(const Fp32TileParams* __restrict__ series,
                                                         int nseries, int64_t total,
                                                         unsigned long long* __restrict__ counter) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long t0 = 0;
        if (lane == 0) t0 = atomicAdd(counter, 1ull);
        const int64_t tt = (int64_t)__shfl_sync(kFullMask, t0, 0);
        if (tt >= total) break;
        int lo = 0, hi = nseries - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (series[mid].tile_begin <= tt) lo = mid;
            else hi = mid - 1;
        }
        const Fp32TileParams P = series[lo];
        if (!P.hazard) continue;
        int64_t band, seg;
        if (fp32_tile_of(P, tt - P.tile_begin + P.tile_skip, 32 * R, band, seg)) tile_guard<R>(P, band, seg, lane);
    }
}

}  // namespace

// Van Herk / Gil-Werman sliding minimum, part 1: prefix and suffix minima of
// the inverse norms within blocks of `blk` windows (NaN, a flat window, is
// ignored by fmin).
__global__ void hazard_block_minima_kernel(const double* __restrict__ nn, int64_t PL, int64_t blk,
                                           double* __restrict__ pre, double* __restrict__ suf) {
    hazard_block_minima(nn, PL, blk, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, pre, suf);
}

// Part 2: flag[w + 1] = 1 when window w is a hazard: flat, or its inverse norm
// exceeds kGuardRatio times the smallest inverse norm among windows
// [w - look, w] (look = blk - 1).  flag[0] = 0; an inclusive scan then turns
// flag into prefix counts.
__global__ void hazard_flags_kernel(const double* __restrict__ nn, const double* __restrict__ pre,
                                    const double* __restrict__ suf, int64_t PL, int64_t blk,
                                    int* __restrict__ flag) {
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w <= PL;
         w += (int64_t)gridDim.x * blockDim.x) {
        if (w == PL) {
            flag[0] = 0;
            continue;
        }
        flag[w + 1] = hazard_flag(nn, pre, suf, blk, w);
    }
}

// FP64 recurrence terms, the FP32 records' formulas without the rounding to
// float: df[i] = (A[i+m] - A[i]) / 2, dg[i] = (A[i+m] - mean[i+1]) + (A[i] - mean[i]).
__global__ void guard_terms_kernel(const double* __restrict__ A, int64_t m, int64_t PL,
                                   const double* __restrict__ mean, double* __restrict__ df,
                                   double* __restrict__ dg) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < PL;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (i + 1 < PL) {
            const double xin = A[i + m], xout = A[i];
            df[i] = (xin - xout) * 0.5;
            dg[i] = (xin - mean[i + 1]) + (xout - mean[i]);
        } else {
            df[i] = 0.0;
            dg[i] = 0.0;
        }
    }
}

// ---- near-duplicate pass ----------------------------------------------------
// Windows whose best FP32 u lies below the FP32 resolution floor (u formed by
// cancellation carries an absolute error of ~1e-7..1e-6) are collected, their
// keys reset, and every pair among them recomputed exactly: a near-duplicate's
// best partner has a tiny u too, so it is in the same set.

__global__ void neardup_collect_kernel(const unsigned long long* __restrict__ key, int64_t PL,
                                       float tau, unsigned long long init, int* __restrict__ list,
                                       int* __restrict__ count, int cap) {
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < PL;
         w += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = key[w];
        if (k >= init) continue;  // no neighbour
        if (unord_f32((unsigned)(k >> 32)) < tau) {
            const int i = atomicAdd(count, 1);
            if (i < cap) list[i] = (int)w;
        }
    }
}

__global__ void neardup_reset_kernel(const int* __restrict__ list, int count,
                                     unsigned long long* __restrict__ key, unsigned long long init) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        key[list[i]] = init;
}

// Tile (ti, tj) of the list x list pair square, 32 x 32 pairs, 2 x 2 per
// thread: centred FP64 dot products, u = 1 - dot * nn_w * nn_v, min-merged
// into the row window's key (the square holds both orders of every pair).
__global__ void __launch_bounds__(256) neardup_pairs_kernel(const NearDupParams P) {
    constexpr int TB = 32, KC = 32;
    __shared__ double sr[TB][KC + 1];
    __shared__ double sc[TB][KC + 1];
    __shared__ unsigned long long rmin[TB][16];
    const int64_t nt = (P.count + TB - 1) / TB;
    const int64_t ti = blockIdx.x / nt, tj = blockIdx.x % nt;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    for (int64_t k0 = 0; k0 < P.m; k0 += KC) {
        __syncthreads();
        for (int e = threadIdx.x; e < TB * KC; e += blockDim.x) {
            const int q = e / KC, kk = e % KC;
            const int64_t k = k0 + kk;
            const int64_t ir = ti * TB + q, ic = tj * TB + q;
            double vr = 0.0, vc = 0.0;
            if (k < P.m && ir < P.count) {
                const int64_t w = P.list[ir];
                vr = P.A[w + k] - P.mean[w];
            }
            if (k < P.m && ic < P.count) {
                const int64_t v = P.list[ic];
                vc = P.A[v + k] - P.mean[v];
            }
            sr[q][kk] = vr;
            sc[q][kk] = vc;
        }
        __syncthreads();
        const int kn = (int)min((int64_t)KC, P.m - k0);
        for (int kk = 0; kk < kn; ++kk) {
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int c = 0; c < 2; ++c)
                    acc[a][c] = __fma_rn(sr[ty * 2 + a][kk], sc[tx * 2 + c][kk], acc[a][c]);
        }
    }
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int64_t ir = ti * TB + ty * 2 + a;
        unsigned long long best = kNoKey;
        if (ir < P.count) {
            const int64_t w = P.list[ir];
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int64_t ic = tj * TB + tx * 2 + c;
                if (ic >= P.count) continue;
                const int64_t v = P.list[ic];
                const int64_t g = w > v ? w - v : v - w;
                if (g < P.g_lo || g >= P.g_hi) continue;
                const double u = __fma_rn(-acc[a][c], P.norm[w] * P.norm[v], 1.0);
                const float fu = (float)u;
                if (fu < P.ulim) {
                    const unsigned long long kk = guard_key(fu, v);
                    best = kk < best ? kk : best;
                }
            }
        }
        rmin[ty * 2 + a][tx] = best;
    }
    __syncthreads();
    if (threadIdx.x < TB) {
        const int64_t ir = ti * TB + threadIdx.x;
        unsigned long long best = kNoKey;
        for (int x = 0; x < 16; ++x) best = rmin[threadIdx.x][x] < best ? rmin[threadIdx.x][x] : best;
        if (ir < P.count && best != kNoKey) atomicMin(P.key + P.list[ir], best);
    }
}

template <int R>
void launch_fp64_guard(const Fp32TileParams* series_dev, int nseries, int64_t total,
                       unsigned long long* counter, cudaStream_t s) {
    const int64_t want = (total + 3) / 4;
    const int64_t blocks = std::min<int64_t>(want, (int64_t)sm_count() * 8);
    if (blocks > 0) fp64_guard_kernel<R><<<(unsigned)blocks, 128, 0, s>>>(series_dev, nseries, total, counter);
}

template void launch_fp64_guard<8>(const Fp32TileParams*, int, int64_t, unsigned long long*,
                                   cudaStream_t);

}  // namespace mpgpu
