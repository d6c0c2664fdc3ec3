// Device helpers shared by the single-series and batched preparation kernels.
#pragma once

#include "mp_common.cuh"

namespace mpgpu {

// Welford over the chunk `t` of `chunk` consecutive windows: a full Welford
// pass for the chunk's first window, then the sliding update
//   mean' = mean + (x_in - x_out)/m
//   M2'   = M2 + (x_in - x_out)*(x_in - mean' + x_out - mean).
// Writes mean (FP64) and norm = 1/sqrt(M2) (FP64; NaN for a window whose
// values are all equal -- nchg counts value changes -- so every correlation
// with it is NaN, the reference's zero-variance convention).
__device__ __forceinline__ void welford_chunk(const double* __restrict__ A, int64_t m, int64_t PL,
                                              int64_t chunk, int64_t t, const int* __restrict__ nchg,
                                              double* __restrict__ mean_out,
                                              double* __restrict__ norm_out) {
    const int64_t i0 = t * chunk;
    const int64_t i1 = min(PL, i0 + chunk);
    double mean = 0.0, M2 = 0.0;
    for (int64_t k = 0; k < m; ++k) {
        const double x = A[i0 + k];
        const double delta = x - mean;
        mean += delta / (double)(k + 1);
        M2 += delta * (x - mean);
    }
    const double inv_m = 1.0 / (double)m;
    for (int64_t i = i0; i < i1; ++i) {
        if (i > i0) {
            const double xin = A[i + m - 1], xout = A[i - 1];
            const double mnew = mean + (xin - xout) * inv_m;
            M2 += (xin - xout) * (xin - mnew + xout - mean);
            mean = mnew;
        }
        const bool flat = (nchg[i + m - 1] - nchg[i]) == 0;
        mean_out[i] = mean;
        norm_out[i] = (flat || !(M2 > 0.0)) ? __longlong_as_double(0x7ff8000000000000ll)
                                            : 1.0 / sqrt(M2);
    }
}

// FP32 records.  For window i (i < PL):
//   df[i] = (A[i+m] - A[i]) / 2,  dg[i] = (A[i+m] - mean[i+1]) + (A[i] - mean[i])
// (zero for the last window, whose successor does not exist), nn[i] = norm[i].
// Row records are stored as pairs (x[j], x[j+H]) for the f32x2 datapath:
//   rowrec[j] = {df[j], df[j+H], dg[j], dg[j+H], nn[j], nn[j+H], 1, 1}
// Column records duplicate and negate the column terms:
//   colrec[p] = {-df[p], -df[p], -dg[p], -dg[p], nn[p], nn[p], 0, 0}
// Entries past PL read as df = dg = 0, nn = NaN.
__device__ __forceinline__ void fp32_terms(const double* A, int64_t m, int64_t PL,
                                           const double* mean, const double* norm, int64_t i,
                                           float& df, float& dg, float& nn) {
    if (i >= PL) {
        df = 0.f;
        dg = 0.f;
        nn = __int_as_float(0x7fffffff);
        return;
    }
    if (i + 1 < PL) {
        const double xin = A[i + m], xout = A[i];
        df = (float)((xin - xout) * 0.5);
        dg = (float)((xin - mean[i + 1]) + (xout - mean[i]));
    } else {
        df = 0.f;
        dg = 0.f;
    }
    nn = (float)norm[i];
}

__device__ __forceinline__ void pack_fp32_record(const double* A, int64_t m, int64_t PL, int H,
                                                 const double* mean, const double* norm, int64_t j,
                                                 float4* rowrec, float4* colrec) {
    float df0, dg0, nn0, df1, dg1, nn1;
    fp32_terms(A, m, PL, mean, norm, j, df0, dg0, nn0);
    fp32_terms(A, m, PL, mean, norm, j + H, df1, dg1, nn1);
    rowrec[2 * j] = make_float4(df0, df1, dg0, dg1);
    rowrec[2 * j + 1] = make_float4(nn0, nn1, 1.f, 1.f);
    colrec[2 * j] = make_float4(-df0, -df0, -dg0, -dg0);
    colrec[2 * j + 1] = make_float4(nn0, nn0, 0.f, 0.f);
}

}  // namespace mpgpu
