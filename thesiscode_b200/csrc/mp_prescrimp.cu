// PreSCRIMP: the anytime front end of SCRIMP++ (scrimppp/src/ScrimpppOrig.cpp:130-266).
//
// Query windows i = 0, s, 2s, ... (s = floor(stride * m)) each get their whole
// distance profile; every cell updates both windows' profile entries; then,
// from each query's best neighbour j, the diagonal j - i is walked s - 1 cells
// forward and backward with the reference's running dot product.  The
// reference computes the query rows by FFT convolution (FFTW); here each cell
// is a direct FP64 dot product over the window, tiled so that a CTA serves 32
// queries x 256 windows from shared memory (m DFMA per cell, no FFT, and more
// accurate than the FFT's rounding).  All updates are min-merges of 64-bit
// keys, so the result does not depend on the (shuffled, in the reference)
// query order.
#include <cfloat>

#include "mp_common.cuh"
#include "mp_kernels.h"

namespace mpgpu {

namespace {

constexpr int kQB = 32;    // queries per CTA
constexpr int kQT = kQB / 4;  // queries per thread
constexpr int kJB = 256;   // windows per CTA
constexpr int kKC = 32;    // window elements per shared-memory stage
constexpr unsigned long long kNone = ~0ull;

// Distance keys: ord(d) min-merged (exact); index keys: ord(d) with its low
// idx_bits replaced by the neighbour, min-merged (smallest neighbour among
// distances equal to ~2^-(52-idx_bits+12) relative).
__device__ __forceinline__ void merge(unsigned long long* kex, unsigned long long* kix, int64_t w,
                                      double d, int64_t nb, int idx_bits) {
    const unsigned long long o = ord_f64(d);
    const unsigned long long low = (1ull << idx_bits) - 1ull;
    atomicMin(kex + w, o);
    atomicMin(kix + w, (o & ~low) | (unsigned long long)nb);
}

// The reference's distance of one cell (ScrimpppOrig.cpp:195, 226, 246):
// 2 * (m - (qt - m * mean_j * mean_i) / (sigma_j * sigma_i)), same operation order.
__device__ __forceinline__ double orig_distance(double mm, double qt, double mean_j, double mean_i,
                                                double sig_j, double sig_i) {
    const double corr = __dmul_rn(__dmul_rn(mm, mean_j), mean_i);
    const double x = __ddiv_rn(__dsub_rn(qt, corr), __dmul_rn(sig_j, sig_i));
    return __dmul_rn(2.0, __dsub_rn(mm, x));
}

}  // namespace

// ScrimpppOrig.cpp:86-107: window sums as prefix-sum differences, mean,
// variance S2/m - mean^2 and sigma = sqrt(variance).
__global__ void orig_stats_kernel(const double* __restrict__ cs, const double* __restrict__ cs2,
                                  int64_t PL, int64_t m, double* __restrict__ mean,
                                  double* __restrict__ sigma) {
    const double mm = (double)m;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < PL;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double s = i == 0 ? cs[m - 1] : __dsub_rn(cs[m - 1 + i], cs[i - 1]);
        const double s2 = i == 0 ? cs2[m - 1] : __dsub_rn(cs2[m - 1 + i], cs2[i - 1]);
        const double mu = __ddiv_rn(s, mm);
        mean[i] = mu;
        sigma[i] = __dsqrt_rn(__dsub_rn(__ddiv_rn(s2, mm), __dmul_rn(mu, mu)));
    }
}

__global__ void prescrimp_keys_init_kernel(unsigned long long* __restrict__ a, int64_t count) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        a[i] = kNone;
}

// Query rows: CTA b covers windows [wt*256, wt*256+256) and queries
// [qt*32, qt*32+32), wt = b % window tiles, qt = b / window tiles (a 1-D grid,
// so any number of queries fits).  Thread (ty, tx) accumulates 8 queries x 4
// windows (12 shared-memory reads per 32 FMAs).
__global__ void __launch_bounds__(256) prescrimp_rows_kernel(const PreScrimpParams P) {
    __shared__ double sq[kQB][kKC + 1];
    __shared__ double sw[kJB + kKC];
    __shared__ double cbest[4][kJB];
    __shared__ int cidx[4][kJB];
    __shared__ double rbest[64][kQB + 1];
    __shared__ int ridx[64][kQB + 1];
    const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;
    const int64_t nwt = (P.PL + kJB - 1) / kJB;
    const int64_t j0 = ((int64_t)blockIdx.x % nwt) * kJB;
    const int64_t t0 = ((int64_t)blockIdx.x / nwt) * kQB;
    double acc[kQT][4];
#pragma unroll
    for (int r = 0; r < kQT; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
    for (int64_t k0 = 0; k0 < P.m; k0 += kKC) {
        __syncthreads();
        for (int e = threadIdx.x; e < kQB * kKC; e += blockDim.x) {
            const int qi = e / kKC, kk = e % kKC;
            const int64_t t = t0 + qi, k = k0 + kk;
            sq[qi][kk] = (t < P.Q && k < P.m) ? P.A[t * P.step + k] : 0.0;
        }
        for (int e = threadIdx.x; e < kJB + kKC; e += blockDim.x) {
            const int64_t x = j0 + k0 + e;
            sw[e] = x < P.n ? P.A[x] : 0.0;  // zero past the series: only cells j >= PL read it
        }
        __syncthreads();
        const int kn = (int)min((int64_t)kKC, P.m - k0);
        for (int kk = 0; kk < kn; ++kk) {
            double a[kQT], w[4];
#pragma unroll
            for (int r = 0; r < kQT; ++r) a[r] = sq[ty * kQT + r][kk];
#pragma unroll
            for (int c = 0; c < 4; ++c) w[c] = sw[tx * 4 + c + kk];
#pragma unroll
            for (int r = 0; r < kQT; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = __fma_rn(a[r], w[c], acc[r][c]);
        }
    }
    // distances; per window the best of this thread's 4 queries, per query the
    // best of its 4 windows
    const double mm = (double)P.m;
    double cb[4], rb[kQT];
    int ci[4], ri[kQT];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        cb[c] = DBL_MAX;
        ci[c] = -1;
    }
#pragma unroll
    for (int r = 0; r < kQT; ++r) {
        rb[r] = DBL_MAX;
        ri[r] = -1;
    }
#pragma unroll
    for (int r = 0; r < kQT; ++r) {
        const int64_t t = t0 + ty * kQT + r;
        if (t >= P.Q) continue;
        const int64_t i = t * P.step;
        const double mi = P.mean[i], si = P.sigma[i];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int64_t j = j0 + tx * 4 + c;
            if (j >= P.PL) continue;
            if (j > i - P.excl && j < i + P.excl) continue;  // ScrimpppOrig.cpp:190-193
            const double d = orig_distance(mm, acc[r][c], P.mean[j], mi, P.sigma[j], si);
            if (d < cb[c]) {
                cb[c] = d;
                ci[c] = (int)i;
            }
            if (d < rb[r]) {
                rb[r] = d;
                ri[r] = (int)j;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        cbest[ty][tx * 4 + c] = cb[c];
        cidx[ty][tx * 4 + c] = ci[c];
    }
#pragma unroll
    for (int r = 0; r < kQT; ++r) {
        rbest[tx][ty * kQT + r] = rb[r];
        ridx[tx][ty * kQT + r] = ri[r];
    }
    __syncthreads();
    // windows: one thread per window of the tile
    {
        const int c = threadIdx.x;
        double b = cbest[0][c];
        int bi = cidx[0][c];
        for (int y = 1; y < 4; ++y)
            if (cidx[y][c] >= 0 && (bi < 0 || cbest[y][c] < b)) {
                b = cbest[y][c];
                bi = cidx[y][c];
            }
        if (bi >= 0) merge(P.kex, P.kix, j0 + c, b, bi, P.idx_bits);
    }
    // queries: the first 32 threads
    if (threadIdx.x < kQB) {
        const int q = threadIdx.x;
        const int64_t t = t0 + q;
        if (t < P.Q) {
            double b = DBL_MAX;
            int bi = -1;
            for (int x = 0; x < 64; ++x)
                if (ridx[x][q] >= 0 && (bi < 0 || rbest[x][q] < b)) {
                    b = rbest[x][q];
                    bi = ridx[x][q];
                }
            if (bi >= 0) {
                merge(P.rex, P.rix, t, b, bi, P.idx_bits);               // the row's own best
                merge(P.kex, P.kix, t * P.step, b, bi, P.idx_bits);      // profile[i]
            }
        }
    }
}

// Diagonal walks from each query's best neighbour (ScrimpppOrig.cpp:212-255):
// thread 2t walks forward, 2t+1 backward, s - 1 cells each.
__global__ void prescrimp_refine_kernel(const PreScrimpParams P) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t t = g >> 1;
    if (t >= P.Q) return;
    const bool fwd = (g & 1) == 0;
    const unsigned long long rx = P.rex[t];
    if (rx == kNone) return;
    const unsigned long long low = (1ull << P.idx_bits) - 1ull;
    const int64_t i = t * P.step;
    const int64_t j = (int64_t)(P.rix[t] & low);
    const double dmin = unord_f64(rx);
    const double mm = (double)P.m;
    const double* A = P.A;
    // lastz = (m - profile[i] / 2) * (sigma_j * sigma_i) + m * mean_j * mean_i
    double z = __dadd_rn(__dmul_rn(__dsub_rn(mm, __ddiv_rn(dmin, 2.0)),
                                   __dmul_rn(P.sigma[j], P.sigma[i])),
                         __dmul_rn(__dmul_rn(mm, P.mean[j]), P.mean[i]));
    if (fwd) {
        for (int64_t k = 1; k < P.step && i + k < P.PL && j + k < P.PL; ++k) {
            z = __dadd_rn(__dsub_rn(z, __dmul_rn(A[i + k - 1], A[j + k - 1])),
                          __dmul_rn(A[i + k + P.m - 1], A[j + k + P.m - 1]));
            const double d = orig_distance(mm, z, P.mean[j + k], P.mean[i + k], P.sigma[j + k],
                                           P.sigma[i + k]);
            if (d < DBL_MAX) {  // NaN and +inf never lower an entry (the reference's '<')
                merge(P.kex, P.kix, i + k, d, j + k, P.idx_bits);
                merge(P.kex, P.kix, j + k, d, i + k, P.idx_bits);
            }
        }
    } else {
        for (int64_t k = 1; k < P.step && i - k >= 0 && j - k >= 0; ++k) {
            z = __dadd_rn(__dsub_rn(z, __dmul_rn(A[i - k + P.m], A[j - k + P.m])),
                          __dmul_rn(A[i - k], A[j - k]));
            const double d = orig_distance(mm, z, P.mean[j - k], P.mean[i - k], P.sigma[j - k],
                                           P.sigma[i - k]);
            if (d < DBL_MAX) {
                merge(P.kex, P.kix, i - k, d, j - k, P.idx_bits);
                merge(P.kex, P.kix, j - k, d, i - k, P.idx_bits);
            }
        }
    }
}

// Keys -> squared distances (the reference's "distance") and indices; windows
// no cell reached keep the reference's initial values (+inf, 0).
__global__ void prescrimp_finalize_kernel(const unsigned long long* __restrict__ kex,
                                          const unsigned long long* __restrict__ kix, int64_t PL,
                                          int idx_bits, double* __restrict__ d2,
                                          int64_t* __restrict__ idx) {
    const unsigned long long low = (1ull << idx_bits) - 1ull;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < PL;
         i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long e = kex[i];
        if (e == kNone) {
            d2[i] = __longlong_as_double(0x7ff0000000000000ll);
            idx[i] = 0;
        } else {
            d2[i] = unord_f64(e);
            idx[i] = (int64_t)(kix[i] & low);
        }
    }
}

void launch_prescrimp(const PreScrimpParams& P, cudaStream_t s) {
    const int64_t tiles = ((P.PL + kJB - 1) / kJB) * ((P.Q + kQB - 1) / kQB);
    prescrimp_rows_kernel<<<(unsigned)tiles, 256, 0, s>>>(P);
    const int64_t threads = 2 * P.Q;
    prescrimp_refine_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(P);
}

}  // namespace mpgpu
