// Shared device-side definitions of the mpgpu library (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cmath>
#include <cstring>

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "mpgpu is written for sm_100a (B200) only"
#endif

namespace mpgpu {

constexpr unsigned kFullMask = 0xffffffffu;

// ---------------------------------------------------------------------------
// Host helpers shared by the entry points.
// ---------------------------------------------------------------------------

// Monotone map float -> uint32 on the host (the same map as ord_f32).
inline unsigned host_ord_f32(float v) {
    unsigned b;
    std::memcpy(&b, &v, 4);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Sub-buffers of a scratch arena start on 256-byte boundaries.
constexpr size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Where a caller's buffer lives, seen from device `device`: host memory
// (pageable or pinned), memory the kernels on `device` may address (its own
// device memory, or managed memory), or device memory of another GPU, which
// the entry points refuse: a kernel on `device` would need peer access to
// touch it, and without that the access faults.
enum class MemSpace { Host, Device, OtherDevice };
inline MemSpace mem_space(const void* p, int device) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return MemSpace::Host;
    }
    if (at.type == cudaMemoryTypeManaged) return MemSpace::Device;
    if (at.type == cudaMemoryTypeDevice)
        return at.device == device ? MemSpace::Device : MemSpace::OtherDevice;
    return MemSpace::Host;
}

// Streaming multiprocessors of the current device (148 on a B200), read once
// per device; persistent and grid-stride launches are sized in multiples of
// it.  A failed query answers with the B200's count.
inline int sm_count() {
    constexpr int kB200Sms = 148;
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return kB200Sms;
    }
    if (dev < 0 || dev >= 64) return kB200Sms;
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
        cudaGetLastError();
        return kB200Sms;
    }
    cached[dev].store(v, std::memory_order_relaxed);
    return v;
}

// Grid of a grid-stride launch of 256-thread blocks over `count` items: one
// block per 256 items, at most 32 blocks per SM.
inline unsigned grid_for(int64_t count) {
    int64_t b = (count + 255) / 256;
    if (b < 1) b = 1;
    const int64_t cap = (int64_t)sm_count() * 32;
    return (unsigned)(b > cap ? cap : b);
}

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

// Bit pattern of a double, on the host or the device.
__host__ __device__ __forceinline__ long long f64_bits(double v) {
#ifdef __CUDA_ARCH__
    return __double_as_longlong(v);
#else
    long long b;
    std::memcpy(&b, &v, sizeof b);
    return b;
#endif
}

// FP64 form, index key.  The low idx_bits hold (2^idx_bits - 1 - neighbour),
// so that among equal high parts a max picks the smaller neighbour.  The high
// 64 - idx_bits bits order candidates by v = m - score (half the squared
// distance; exact by Sterbenz for score in [m/2, 2m]), smaller v higher: a
// region bit (set for v <= 0) and then |v|'s bits taken relative to
// vlo = 2^(t-64), where the host picks t with 2^t > 2m + 2, so that 64
// binades need 6 exponent bits instead of 11 and the freed bits keep mantissa
// (33 mantissa bits at idx_bits = 24: candidates closer than ~1.2e-10 in
// relative squared distance share a high part).  For v > 0, |v| outside
// [vlo, 2^t) clamps to the range ends (no candidate above the floor score -1
// has v >= 2^t).  For v <= 0 (score >= m) the first 32 binades [vlo, 2^(t-32))
// keep that resolution -- scores a rounding error above m land there -- and
// every larger |v| up to inf (scores far above m, from the huge sInv of a
// window whose variance rounds to a tiny positive value) goes to a coarser
// region above them: all 11 exponent bits and 51 - idx_bits mantissa bits, so
// the key stays monotone in the score over the whole double range.
__host__ __device__ __forceinline__ unsigned long long idx_key_f64(double score, double m,
                                                                   unsigned long long neighbour,
                                                                   int idx_bits, long long vlo_bits) {
    const unsigned long long lowmask = (1ull << idx_bits) - 1ull;
    const int shift = idx_bits > 5 ? idx_bits - 5 : 0;
    const long long span = 1ll << 58;  // 64 binades of 2^52 bit patterns
    const long long fine = 1ll << 57;  // 32 binades
    const double v = m - score;
    long long x = f64_bits(fabs(v)) - vlo_bits;
    x = x < 0 ? 0 : x;
    unsigned long long field;
    if (v > 0.0) {
        field = (unsigned long long)(span - 1 - (x > span - 1 ? span - 1 : x)) >> shift;
    } else {
        const unsigned long long low =
            x < fine ? (unsigned long long)x >> shift
                     : (1ull << (62 - idx_bits)) | ((unsigned long long)(x - fine) >> (idx_bits + 1));
        field = (1ull << (63 - idx_bits)) | low;
    }
    return (field << idx_bits) | (lowmask - neighbour);
}

// Host side of the index key: vlo_bits = the bit pattern of 2^(t-64), with
// 2^t > 2m + 2 >= every half squared distance m - score of a candidate whose
// correlation is at least -1; idx_bits = bits that hold every neighbour index
// up to maxval.
inline long long key_vlo_bits(int64_t m) {
    int t = 1;
    while (t < 62 && std::ldexp(1.0, t) <= 2.0 * (double)m + 2.0) ++t;
    return (long long)(1023 + t - 64) << 52;
}
inline int bits_for(uint64_t maxval) {
    int b = 1;
    while (b < 63 && (1ull << b) <= maxval) ++b;
    return b;
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

// ---------------------------------------------------------------------------
// Per-warp ring of 32-byte row records in shared memory.
//
// Lane l of a band reads record base + 8*l + k while the other lanes read
// theirs, i.e. 32 records 8 apart.  Read straight from global memory those hit
// 32 cache lines per instruction; staged here they come in with coalesced
// 16-byte loads and go out conflict-free: slot s lives at byte
//   off(s) = 32*s + 16*(s >> 3),
// a 16-byte gap after every 8 records, so the eight lanes of a quarter-warp
// (records 8 apart, 272 bytes apart) start in eight distinct 16-byte bank
// groups (a wrap moves a slot by 320 records = 680 chunks, a multiple of 8,
// so it keeps its group).  Slots 320..327 mirror slots 0..7, so the 8
// consecutive records a lane reads in one chunk never wrap: their offsets are
// the chunk's base plus compile-time constants.
// ---------------------------------------------------------------------------
constexpr int kRecRing = 320;  // records per warp ring (multiple of 8, >= 33*8 + 16)
constexpr int kRecMirror = 8;
constexpr int kRecRingBytes = 32 * (kRecRing + kRecMirror) + 16 * ((kRecRing + kRecMirror) / 8);

__device__ __forceinline__ int rec_off(int slot) { return 32 * slot + 16 * (slot >> 3); }

// Offset of record (s0 + b) given off(s0) and C = s0 % 8 (both b and C
// compile-time), valid for s0 < kRecRing and b < kRecMirror.
template <int C>
__device__ __forceinline__ constexpr int rec_step(int b) {
    return 32 * b + 16 * ((C + b) >> 3);
}

// Writes 16-byte half `half` of record t (and its mirror).
__device__ __forceinline__ int rec_slot(int t) { return t % kRecRing; }
__device__ __forceinline__ void rec_store(char* ring, int t, int half, uint4 v) {
    const int s = rec_slot(t);
    *reinterpret_cast<uint4*>(ring + rec_off(s) + 16 * half) = v;
    if (s < kRecMirror) *reinterpret_cast<uint4*>(ring + rec_off(s + kRecRing) + 16 * half) = v;
}
__device__ __forceinline__ uint4 lds128(const char* p) { return *reinterpret_cast<const uint4*>(p); }
__device__ __forceinline__ uint2 lds64(const char* p) { return *reinterpret_cast<const uint2*>(p); }

}  // namespace mpgpu
