// Shared device-side definitions of the mpgpu library (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "mpgpu is written for sm_100a (B200) only"
#endif

namespace mpgpu {

constexpr unsigned kFullMask = 0xffffffffu;

// ---------------------------------------------------------------------------
// Keys.  A profile entry is merged across threads, warps and CTAs with plain
// 64-bit integer max (FP64 form) or min (FP32 form) atomics, so every
// candidate is first mapped to an integer that orders like its value.
// ---------------------------------------------------------------------------

// Monotone map double -> uint64 (larger double -> larger key).  NaN never
// reaches a key: callers only flush scores that passed `score > -1.0`.
__device__ __forceinline__ unsigned long long ord_f64(double v) {
    const long long b = __double_as_longlong(v);
    return b < 0 ? ~(unsigned long long)b : ((unsigned long long)b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord_f64(unsigned long long k) {
    const long long b = (k & 0x8000000000000000ull) ? (long long)(k & 0x7fffffffffffffffull)
                                                    : (long long)~k;
    return __longlong_as_double(b);
}
// Monotone map float -> uint32 (larger float -> larger key).
__device__ __forceinline__ unsigned ord_f32(float v) {
    const unsigned b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unord_f32(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// FP64 form, index key: the top (64 - idx_bits) bits order like the distance
// proxy t = score - m (exact by Sterbenz for score in [m/2, 2m]); the low
// idx_bits hold (2^idx_bits - 1 - neighbour) so that a max picks the larger
// score and, among scores whose truncated t agree, the smaller neighbour.
__device__ __forceinline__ unsigned long long idx_key_f64(double score, double m,
                                                          unsigned long long neighbour,
                                                          int idx_bits) {
    const unsigned long long lowmask = (1ull << idx_bits) - 1ull;
    const unsigned long long hi = ord_f64(score - m) & ~lowmask;
    return hi | (lowmask - neighbour);
}

// ---------------------------------------------------------------------------
// Packed FP32 helpers (Blackwell f32x2 datapath).  A float2 pair lives in one
// 64-bit register pair; one instruction performs both lanes' operations.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_unpack(unsigned long long v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long f2_mul(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Bounded-work guard: device loops that wait on nothing but their own data
// need no limit; this library has no cross-CTA waits at all.

}  // namespace mpgpu
