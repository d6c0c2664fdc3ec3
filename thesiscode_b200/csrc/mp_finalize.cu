// Key initialisation and finalisation: merged 64-bit keys -> squared
// distances and neighbour indices (ScrimpVertBlocked.cpp:171-174 applies
// d2 = 2m - 2*score to the final scores).
#include "mp_common.cuh"
#include "mp_kernels.h"

namespace mpgpu {

__global__ void init_keys_kernel(unsigned long long* __restrict__ k, int64_t count,
                                 unsigned long long v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x)
        k[i] = v;
}

// FP64 form.  kexact/kidx start at 0 in every shard; a window improved by some
// pair has an exact key above ord(-1.0).  Untouched windows keep score -1 and
// neighbour 0, the reference's initial values (ScrimpVertBlocked.cpp:103-104).
__global__ void finalize_fp64_kernel(const unsigned long long* __restrict__ kexact,
                                     const unsigned long long* __restrict__ kidx,
                                     int64_t key_stride, int shards, int64_t PL, double m,
                                     int idx_bits, double* __restrict__ d2,
                                     int64_t* __restrict__ idx) {
    const unsigned long long floor_key = ord_f64(-1.0);
    const unsigned long long lowmask = (1ull << idx_bits) - 1ull;
    const double twice_m = __dmul_rn(2.0, m);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < PL;
         i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long ke = 0, ki = 0;
        for (int s = 0; s < shards; ++s) {
            ke = max(ke, kexact[(int64_t)s * key_stride + i]);
            ki = max(ki, kidx[(int64_t)s * key_stride + i]);
        }
        double score = -1.0;
        int64_t nb = 0;
        if (ke > floor_key) {
            score = unord_f64(ke);
            nb = (int64_t)(lowmask - (ki & lowmask));
        }
        d2[i] = __dsub_rn(twice_m, __dmul_rn(2.0, score));
        idx[i] = nb;
    }
}

// FP32 form.  key = (ord(u) << 32) | neighbour, min-merged; the initial key
// encodes u = 1 + 1/m (score -1) with neighbour 0.  refine != 0 recomputes the
// chosen pair's distance from a centred FP64 dot product.
__global__ void finalize_fp32_kernel(const unsigned long long* __restrict__ key, int64_t PL,
                                     double m, const double* __restrict__ A,
                                     const double* __restrict__ mean,
                                     const double* __restrict__ norm, int refine,
                                     double* __restrict__ d2, int64_t* __restrict__ idx) {
    const float ulim = (float)(1.0 + 1.0 / m);
    const unsigned long long init = (unsigned long long)ord_f32(ulim) << 32;
    const int64_t mm = (int64_t)m;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < PL;
         i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = key[i];
        if (k >= init) {
            d2[i] = 2.0 * m + 2.0;
            idx[i] = 0;
            continue;
        }
        const int64_t j = (int64_t)(k & 0xffffffffull);
        idx[i] = j;
        if (refine) {
            const double mi = mean[i], mj = mean[j];
            double c = 0.0;
            for (int64_t t = 0; t < mm; ++t) c = __fma_rn(A[i + t] - mi, A[j + t] - mj, c);
            d2[i] = 2.0 * m * (1.0 - c * norm[i] * norm[j]);
        } else {
            d2[i] = 2.0 * m * (double)unord_f32((unsigned)(k >> 32));
        }
    }
}

// Guarded FP32 form: keys as finalize_fp32_kernel's, except that the FP32
// pass's keys name candidate groups (kFp32GroupBit); each resolves to the
// best of its candidates and kPickSpan more on each side, in FP64
// (fp32_pick_neighbour), within the join's diagonals [g_lo, g_hi).  Every
// distance is the chosen pair's, from a centred FP64 dot product.
__global__ void finalize_fp32_guarded_kernel(const unsigned long long* __restrict__ key, int64_t PL,
                                             double m, const double* __restrict__ A,
                                             const double* __restrict__ mean,
                                             const double* __restrict__ norm, int64_t g_lo,
                                             int64_t g_hi, double* __restrict__ d2,
                                             int64_t* __restrict__ idx) {
    const float ulim = (float)(1.0 + 1.0 / m);
    const unsigned long long init = (unsigned long long)ord_f32(ulim) << 32;
    const int64_t mm = (int64_t)m;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < PL;
         i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = key[i];
        if (k >= init) {
            d2[i] = 2.0 * m + 2.0;
            idx[i] = 0;
            continue;
        }
        const unsigned lo = (unsigned)k;
        int64_t j = (int64_t)(lo & ~kFp32GroupBit);
        if (lo & kFp32GroupBit) {
            const int count = (int)((unsigned)(k >> 32) & 7u) + 1;
            const int64_t q = fp32_pick_neighbour(A, mean, norm, mm, PL, g_lo, g_hi, i, j - kPickSpan,
                                                  count + 2 * kPickSpan);
            if (q >= 0) j = q;
        }
        idx[i] = j;
        const double mi = mean[i], mj = mean[j];
        double c = 0.0;
        for (int64_t t = 0; t < mm; ++t) c = __fma_rn(A[i + t] - mi, A[j + t] - mj, c);
        d2[i] = 2.0 * m * (1.0 - c * norm[i] * norm[j]);
    }
}

// Block interface: exact keys start at the caller's current score, index keys
// at 0 (below every candidate).
__global__ void block_keys_init_kernel(const double* __restrict__ prof, int64_t count,
                                       unsigned long long* __restrict__ kexact,
                                       unsigned long long* __restrict__ kidx) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double p = prof[i];
        // a NaN score is never beaten under '>' (the reference's semantics)
        kexact[i] = (p != p) ? ~0ull : ord_f64(p);
        kidx[i] = 0;
    }
}

__global__ void block_finalize_kernel(const unsigned long long* __restrict__ kexact,
                                      const unsigned long long* __restrict__ kidx,
                                      int64_t key_stride, int shards, int64_t count, int idx_bits,
                                      double* __restrict__ prof, int64_t* __restrict__ idx) {
    const unsigned long long lowmask = (1ull << idx_bits) - 1ull;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double p = prof[i];
        if (p != p) continue;
        unsigned long long ke = 0, ki = 0;
        for (int s = 0; s < shards; ++s) {
            ke = max(ke, kexact[(int64_t)s * key_stride + i]);
            ki = max(ki, kidx[(int64_t)s * key_stride + i]);
        }
        if (ke > ord_f64(p)) {
            prof[i] = unord_f64(ke);
            idx[i] = (int64_t)(lowmask - (ki & lowmask));
        }
    }
}

}  // namespace mpgpu
