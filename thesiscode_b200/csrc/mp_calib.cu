// FMA-throughput calibration kernels: the denominators of the join kernels'
// compute roofline (FP32 and FP64 CUDA-core pipes; no tensor cores involved).
// Each thread runs 8 independent fused-multiply-add chains so the pipes, not
// the dependency latency, bound the rate.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/mpgpu.h"
#include "mp_common.cuh"

namespace mpgpu {
namespace {

__global__ void peak_f32x2_kernel(float* out, int iters) {
    float2 a[8];
    const float s = 1.0f + 1e-7f * (float)threadIdx.x;
    const float2 mul = make_float2(0.999999f, 0.999998f);
    const float2 add = make_float2(1e-7f, 2e-7f);
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = make_float2(s + k, s - k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = __ffma2_rn(a[k], mul, add);
    }
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += a[k].x + a[k].y;
    if (acc == 12345.678f) out[threadIdx.x] = acc;
}

__global__ void peak_f32_kernel(float* out, int iters) {
    float a[8];
    const float s = 1.0f + 1e-7f * (float)threadIdx.x;
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = s + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = __fmaf_rn(a[k], 0.999999f, 1e-7f);
    }
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += a[k];
    if (acc == 12345.678f) out[threadIdx.x] = acc;
}

__global__ void peak_f64_kernel(double* out, int iters) {
    double a[8];
    const double s = 1.0 + 1e-9 * (double)threadIdx.x;
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = s + k;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = __fma_rn(a[k], 0.999999, 1e-9);
    }
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += a[k];
    if (acc == 12345.678) out[threadIdx.x] = acc;
}

}  // namespace
}  // namespace mpgpu

// which: 0 = FP32 (scalar FFMA), 1 = FP32 (f32x2 FFMA), 2 = FP64.
extern "C" int mp_measure_fma_peak(int device, int which, double* flops_per_s) {
    using namespace mpgpu;
    if (!flops_per_s || which < 0 || which > 2) return MP_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return MP_ERR_NO_DEVICE;
    void* out = nullptr;
    if (cudaMalloc(&out, 4096) != cudaSuccess) return MP_ERR_OUT_OF_MEMORY;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sm_count() * 8, threads = 256;
    const int iters = (which == 2) ? 2048 : 8192;
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (which == 0) peak_f32_kernel<<<blocks, threads>>>((float*)out, iters);
        else if (which == 1) peak_f32x2_kernel<<<blocks, threads>>>((float*)out, iters);
        else peak_f64_kernel<<<blocks, threads>>>((double*)out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double fmas = (double)blocks * threads * iters * 32.0 * (which == 1 ? 2.0 : 1.0);
        if (rep > 0 && ms > 0.f) best = std::max(best, 2.0 * fmas / (ms * 1e-3));
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return MP_ERR_CUDA;
    *flops_per_s = best;
    return MP_OK;
}
