// C ABI of the mpgpu library (declared in include/mpgpu.h).
//
// Host-side orchestration only: argument checks, device scratch, copies for
// host-resident buffers, and the launch sequence of each entry point.  No
// arithmetic of the profile happens on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpgpu.h"
#include "mp_common.cuh"
#include "mp_kernels.h"
#include "mp_serve.h"

using namespace mpgpu;

struct mp_context {
    int device = 0;
    size_t budget = 0;
    std::string last_error;
    int64_t launches = 0;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    // while a caller's buffer is lent as the scratch (ctx_lend_scratch), the
    // context's own arena waits here
    bool lent = false;
    void* own_arena = nullptr;
    size_t own_bytes = 0;
    bool timing = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double phase_ms[3] = {-1.0, -1.0, -1.0};
    int64_t near_duplicates = -1;  // guarded form: windows of the last near-duplicate pass
};

namespace mpgpu {
size_t ctx_budget(const mp_context* ctx) { return ctx ? ctx->budget : 0; }
int ctx_device(const mp_context* ctx) { return ctx ? ctx->device : 0; }
void ctx_lend_scratch(mp_context* ctx, void* scratch, size_t bytes) {
    if (!ctx) return;
    if (scratch) {
        if (!ctx->lent) {
            ctx->own_arena = ctx->arena;
            ctx->own_bytes = ctx->arena_bytes;
            ctx->lent = true;
        }
        ctx->arena = scratch;
        ctx->arena_bytes = bytes;
    } else if (ctx->lent) {
        ctx->arena = ctx->own_arena;
        ctx->arena_bytes = ctx->own_bytes;
        ctx->own_arena = nullptr;
        ctx->own_bytes = 0;
        ctx->lent = false;
    }
}
}  // namespace mpgpu

namespace {

constexpr int kThreads = 256;
constexpr int64_t kFp64Pad = 64 * 8 + 64;  // records past the end: 32*R + 2R rows, R <= 8
constexpr int kFp32R = 8;
constexpr int64_t kGuardedReanchorK = 512;  // guarded form's default re-anchor interval
constexpr int64_t kFp32Pad = 64 * 8 + 64;

int fail(mp_context* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->last_error = buf;
    return code;
}

#define MP_CUDA(ctx, call)                                                                 \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(ctx, MP_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define MP_LAUNCHED(ctx)                                                                  \
    do {                                                                                  \
        ++(ctx)->launches;                                                                \
        cudaError_t e_ = cudaGetLastError();                                              \
        if (e_ != cudaSuccess)                                                            \
            return fail(ctx, MP_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e_)); \
    } while (0)


// Carves typed sub-buffers out of the context arena.
struct Carve {
    char* base;
    size_t off = 0;
    template <class T>
    T* take(int64_t count) {
        T* p = reinterpret_cast<T*>(base + off);
        off += align_up(sizeof(T) * (size_t)std::max<int64_t>(count, 1));
        return p;
    }
};

int reserve(mp_context* ctx, size_t bytes) {
    if (ctx->budget && bytes > ctx->budget)
        return fail(ctx, MP_ERR_BUDGET, "request needs %zu bytes of device scratch, budget is %zu",
                    bytes, ctx->budget);
    if (bytes <= ctx->arena_bytes) return MP_OK;
    if (ctx->lent)  // a lent scratch is never replaced
        return fail(ctx, MP_ERR_BUDGET, "lent scratch holds %zu bytes, the call needs %zu",
                    ctx->arena_bytes, bytes);
    if (ctx->arena) cudaFree(ctx->arena);
    ctx->arena = nullptr;
    ctx->arena_bytes = 0;
    cudaError_t e = cudaMalloc(&ctx->arena, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, MP_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu) failed: %s", bytes,
                    cudaGetErrorString(e));
    }
    ctx->arena_bytes = bytes;
    return MP_OK;
}


// Key shards spread the 64-bit max reductions of concurrently running bands
// (which all walk the same columns) over more addresses; kept small enough
// (~32 MB of keys) to stay resident in L2.
int fp64_shards(int64_t PL) {
    const double per = 16.0 * (double)PL;
    int64_t s = (int64_t)(32.0e6 / per);
    return (int)std::max<int64_t>(1, std::min<int64_t>(16, s));
}

// Diagonals per lane.  Every band walks all of its columns, so the longest
// band's column count is the critical path whatever R is; R = 8 does the most
// cells per step and was fastest at every size measured on a B200 (FP64 join,
// m = 256: n = 16,384 -> 3.2 ms vs 3.6 ms at R = 4 and 5.2 ms at R = 2, even
// with 63 bands for 148 SMs; n = 524,288 -> 121 vs 190 vs 482 ms).  Only a few
// hundred diagonals (the kernel API's blocks) leave most lanes of an R = 8
// band idle; there narrower bands spread the same steps over more warps.
int pick_fp64_R(int64_t ndiag) {
#ifdef MPGPU_FP64_FORCE_R
    return MPGPU_FP64_FORCE_R;  // tuning builds only
#endif
    if (ndiag >= 2048) return 8;
    if (ndiag >= 512) return 4;
    return ndiag >= 128 ? 2 : 1;
}

int launch_band(int R, const Fp64BandParams& P, cudaStream_t s) {
    switch (R) {
        case 8: launch_fp64_band<8>(P, s); break;
        case 4: launch_fp64_band<4>(P, s); break;
        case 2: launch_fp64_band<2>(P, s); break;
        default: launch_fp64_band<1>(P, s); break;
    }
    return 0;
}

struct Sizes {
    int64_t n, m, PL, excl, lo, hi;
};

int check_join_args(mp_context* ctx, const double* A, int64_t n, int64_t m, int64_t excl,
                    int64_t diag_lo, int64_t diag_hi, double* d2, int64_t* idx, Sizes& S) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    if (!A || !d2 || !idx) return fail(ctx, MP_ERR_INVALID_ARG, "null buffer");
    if (m < 2) return fail(ctx, MP_ERR_INVALID_ARG, "window length m=%lld < 2", (long long)m);
    if (n < m)
        return fail(ctx, MP_ERR_INVALID_ARG,
                    "time series is shorter than the window length (n=%lld, m=%lld)",
                    (long long)n, (long long)m);
    if (n - m + 1 >= (1ll << 31))
        return fail(ctx, MP_ERR_NOT_SUPPORTED, "profile length %lld exceeds 2^31-1",
                    (long long)(n - m + 1));
    S.n = n;
    S.m = m;
    S.PL = n - m + 1;
    S.excl = excl < 0 ? m / 4 : excl;
    S.lo = diag_lo;
    S.hi = diag_hi;
    if (S.lo == 0 && S.hi == 0) {
        S.lo = S.excl + 1;
        S.hi = S.PL;
    }
    S.lo = std::max<int64_t>(S.lo, S.excl + 1);
    S.hi = std::min<int64_t>(S.hi, S.PL);
    if (S.hi < S.lo) S.hi = S.lo;
    return MP_OK;
}

size_t fp64_scratch(int64_t n, int64_t m, int64_t ndiag, bool host_io) {
    const int64_t PL = n - m + 1;
    const int S = fp64_shards(PL);
    size_t b = 0;
    b += align_up(8 * (size_t)(n + 1));          // Apad
    b += 2 * align_up(8 * (size_t)n);            // prefix sums
    b += 2 * align_up(8 * (size_t)PL);           // muS, sInv
    b += align_up(8 * (size_t)std::max<int64_t>(ndiag, 1));  // first QT
    b += align_up(32 * (size_t)(PL + kFp64Pad)); // records
    b += 2 * align_up(8 * (size_t)PL * S);       // keys
    b += align_up(8 * (size_t)(PL + kFp64ThrPad)); // selection thresholds
    if (host_io) b += align_up(8 * (size_t)PL) * 2;
    return b + 4096;
}

// Selection thresholds of the FP64 band join start at -DBL_MAX (every cell
// selects until merges raise them).
unsigned long long no_threshold_bits() {
    const double v = -1.7976931348623157e308;
    unsigned long long b;
    std::memcpy(&b, &v, sizeof b);
    return b;
}

// Guarded form, on top of fp32_scratch: hazard prefix counts and scan
// totals, block minima, FP64 recurrence terms.
// Near-duplicate pass: windows whose best FP32 u is below kNearDupU are
// recomputed pairwise in FP64, at most kNearDupCap of them (cost
// count^2 * m FP64 FMAs; above the cap the FP32 values stand).
constexpr float kNearDupU = 1e-3f;
constexpr int kNearDupCap = 1 << 17;

size_t guard_scratch(int64_t n, int64_t m) {
    const int64_t PL = n - m + 1;
    return align_up(4 * (size_t)(PL + 1)) + align_up(4 * (size_t)((PL + 1 + kThreads - 1) / kThreads + 1)) +
           4 * align_up(8 * (size_t)PL) + align_up(4 * (size_t)kNearDupCap) + 2048;
}

size_t fp32_scratch(int64_t n, int64_t m, bool host_io, size_t nranges = 1) {
    const int64_t PL = n - m + 1;
    size_t b = 0;
    b += align_up(8 * (size_t)(n + kFp32Pad));   // Apad
    b += align_up(4 * (size_t)n);                // change counts
    b += align_up(4 * (size_t)((n + kThreads - 1) / kThreads + 1));
    b += 2 * align_up(8 * (size_t)(PL + kFp32Pad));  // mean, norm
    b += 2 * align_up(32 * (size_t)(PL + kFp32Pad)); // row/col records
    b += align_up(8 * (size_t)PL);               // keys
    b += align_up(sizeof(Fp32TileParams) * std::max<size_t>(nranges, 1)) + 256;  // descriptors, tile counter
    if (host_io) b += align_up(8 * (size_t)PL) * 2;
    return b + 4096;
}

void mark(mp_context* ctx, int k, cudaStream_t st) {
    if (!ctx->timing) return;
    if (!ctx->ev[k]) cudaEventCreate(&ctx->ev[k]);
    cudaEventRecord(ctx->ev[k], st);
}

void collect_phases(mp_context* ctx) {
    for (int k = 0; k < 3; ++k) ctx->phase_ms[k] = -1.0;
    if (!ctx->timing) return;
    for (int k = 0; k < 3; ++k) {
        float ms = 0.f;
        if (ctx->ev[k] && ctx->ev[k + 1] && cudaEventElapsedTime(&ms, ctx->ev[k], ctx->ev[k + 1]) == cudaSuccess)
            ctx->phase_ms[k] = ms;
        else
            cudaGetLastError();
    }
}

}  // namespace

extern "C" {

int mp_set_phase_timing(mp_context* ctx, int on) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    ctx->timing = on != 0;
    return MP_OK;
}

int mp_last_phase_ms(const mp_context* ctx, double* prep_ms, double* join_ms, double* finalize_ms) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    if (prep_ms) *prep_ms = ctx->phase_ms[0];
    if (join_ms) *join_ms = ctx->phase_ms[1];
    if (finalize_ms) *finalize_ms = ctx->phase_ms[2];
    return MP_OK;
}

const char* mp_status_string(int status) {
    switch (status) {
        case MP_OK: return "ok";
        case MP_ERR_INVALID_ARG: return "invalid argument";
        case MP_ERR_OUT_OF_MEMORY: return "out of device memory";
        case MP_ERR_BUDGET: return "request exceeds the memory budget";
        case MP_ERR_CUDA: return "CUDA error";
        case MP_ERR_NOT_SUPPORTED: return "not supported";
        case MP_ERR_NO_DEVICE: return "no usable device";
        case MP_ERR_IO: return "file could not be read or written";
        default: return "unknown status";
    }
}

int mp_context_create(int device, size_t mem_budget_bytes, mp_context** out) {
    if (!out) return MP_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) {
        cudaGetLastError();
        return MP_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) {
        cudaGetLastError();
        return MP_ERR_NO_DEVICE;
    }
    mp_context* c = new mp_context();
    c->device = device;
    c->budget = mem_budget_bytes;
    *out = c;
    return MP_OK;
}

int mp_context_destroy(mp_context* ctx) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    void* own = ctx->lent ? ctx->own_arena : ctx->arena;
    if (own) cudaFree(own);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    delete ctx;
    return MP_OK;
}

const char* mp_last_error(const mp_context* ctx) {
    return ctx ? ctx->last_error.c_str() : "no context";
}

int64_t mp_last_launch_count(const mp_context* ctx) { return ctx ? ctx->launches : -1; }
int64_t mp_last_near_duplicates(const mp_context* ctx) { return ctx ? ctx->near_duplicates : -1; }

size_t mp_selfjoin_scratch_bytes(int64_t n, int64_t m, int precision) {
    if (m < 2 || n < m) return 0;
    if (precision == MP_PREC_FP64) return fp64_scratch(n, m, n - m + 1, true);
    if (precision == MP_PREC_FP32_GUARDED) return fp32_scratch(n, m, true) + guard_scratch(n, m);
    return fp32_scratch(n, m, true);
}

}  // extern "C"

namespace {

struct DiagRange {
    int64_t lo, hi;
};

// The self-join over a list of non-empty diagonal ranges [lo, hi) inside
// [S.lo, S.hi): one preparation, the joins of every range into the same keys,
// one finalisation.
int selfjoin_ranges(mp_context* ctx, const double* A, int64_t n, int64_t m, int precision,
                    int64_t reanchor_k, int64_t blocklen, const Sizes& S,
                    const std::vector<DiagRange>& ranges, double* dist2_out, int64_t* idx_out,
                    void* stream) {
    int rc = MP_OK;
    if (precision != MP_PREC_FP64 && precision != MP_PREC_FP32_REANCHOR &&
        precision != MP_PREC_FP32_GUARDED)
        return fail(ctx, MP_ERR_INVALID_ARG, "unknown precision %d", precision);
    MP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    ctx->launches = 0;
    ctx->near_duplicates = -1;
    const MemSpace sa = mem_space(A, ctx->device), sd = mem_space(dist2_out, ctx->device),
                   si = mem_space(idx_out, ctx->device);
    if (sa == MemSpace::OtherDevice || sd == MemSpace::OtherDevice || si == MemSpace::OtherDevice)
        return fail(ctx, MP_ERR_INVALID_ARG,
                    "A, dist2_out and idx_out must be host memory or device memory of the "
                    "context's device %d", ctx->device);
    const bool a_dev = sa == MemSpace::Device;
    const bool o_dev = sd == MemSpace::Device;
    if ((si == MemSpace::Device) != o_dev)
        return fail(ctx, MP_ERR_INVALID_ARG, "dist2_out and idx_out live in different memory spaces");
    const int64_t PL = S.PL;
    int64_t ndiag = 0;
    for (const DiagRange& r : ranges) ndiag += r.hi - r.lo;
    if (precision == MP_PREC_FP32_GUARDED && ranges.size() > 1)
        return fail(ctx, MP_ERR_NOT_SUPPORTED, "the guarded form takes one diagonal range per call");

    if (precision == MP_PREC_FP64) {
        const int64_t B = blocklen > 0 ? blocklen : 500;
        const int shards = fp64_shards(PL);
        rc = reserve(ctx, fp64_scratch(n, m, ndiag, !o_dev));
        if (rc) return rc;
        Carve cv{(char*)ctx->arena};
        double* Apad = cv.take<double>(n + 1);
        double* cs = cv.take<double>(n);
        double* cs2 = cv.take<double>(n);
        double* muS = cv.take<double>(PL);
        double* sInv = cv.take<double>(PL);
        double* qt0 = cv.take<double>(ndiag);
        double4* rec = cv.take<double4>(PL + kFp64Pad);
        unsigned long long* kex = cv.take<unsigned long long>(PL * shards);
        unsigned long long* kid = cv.take<unsigned long long>(PL * shards);
        double* thr = cv.take<double>(PL + kFp64ThrPad);
        double* d2 = o_dev ? dist2_out : cv.take<double>(PL);
        int64_t* ix = o_dev ? idx_out : cv.take<int64_t>(PL);

        MP_CUDA(ctx, cudaMemcpyAsync(Apad, A, 8 * n, a_dev ? cudaMemcpyDeviceToDevice
                                                           : cudaMemcpyHostToDevice, st));
        mark(ctx, 0, st);
        MP_CUDA(ctx, cudaMemsetAsync(Apad + n, 0, 8, st));
        ref_prefix_kernel<<<1, kPrefixThreads, 0, st>>>(Apad, n, cs, cs2);
        MP_LAUNCHED(ctx);
        ref_stats_kernel<<<grid_for(PL), kThreads, 0, st>>>(cs, cs2, PL, m, muS, sInv);
        MP_LAUNCHED(ctx);
        {
            int64_t off = 0;
            for (const DiagRange& r : ranges) {
                first_qt_kernel<<<grid_for(r.hi - r.lo), kThreads, 0, st>>>(Apad, m, r.lo, r.hi,
                                                                          qt0 + off);
                MP_LAUNCHED(ctx);
                off += r.hi - r.lo;
            }
        }
        MP_CUDA(ctx, cudaMemsetAsync(rec + PL, 0, 32 * kFp64Pad, st));
        pack_fp64_kernel<<<grid_for(PL), kThreads, 0, st>>>(Apad, m, PL, sInv, muS, rec);
        MP_LAUNCHED(ctx);
        MP_CUDA(ctx, cudaMemsetAsync(kex, 0, 8 * (size_t)PL * shards, st));
        MP_CUDA(ctx, cudaMemsetAsync(kid, 0, 8 * (size_t)PL * shards, st));
        init_keys_kernel<<<grid_for(PL + kFp64ThrPad), kThreads, 0, st>>>(
            reinterpret_cast<unsigned long long*>(thr), PL + kFp64ThrPad, no_threshold_bits());
        MP_LAUNCHED(ctx);
        mark(ctx, 1, st);
        int64_t qoff = 0;
        for (const DiagRange& r : ranges) {
            Fp64BandParams P{};
            const int64_t nd = r.hi - r.lo;
            const int R = pick_fp64_R(nd);
            P.colrec = rec;
            P.rowrec = rec;
            P.qt0 = qt0 + qoff;
            qoff += nd;
            P.qt_out = nullptr;
            P.g_lo = r.lo;
            P.g_hi = r.hi;
            P.nbands = (nd + 32 * R - 1) / (32 * R);
            P.blk_origin = S.excl + 1;
            P.B = B;
            P.Tbase = PL;
            P.kexact = kex;
            P.kidx = kid;
            P.key_stride = PL;
            P.shards = shards;
            P.m = (double)m;
            P.floor = -1.0;
            P.idx_bits = bits_for((uint64_t)PL);
            P.key_vlo = key_vlo_bits(m);
            P.thr = thr;
            P.thr_eps = fp64_threshold_eps(P.idx_bits);
            P.thr_tiny = fp64_threshold_tiny(P.m);
            launch_band(R, P, st);
            MP_LAUNCHED(ctx);
        }
        mark(ctx, 2, st);
        finalize_fp64_kernel<<<grid_for(PL), kThreads, 0, st>>>(kex, kid, PL, shards, PL, (double)m,
                                                                bits_for((uint64_t)PL), d2, ix);
        MP_LAUNCHED(ctx);
        mark(ctx, 3, st);
        if (!o_dev) {
            MP_CUDA(ctx, cudaMemcpyAsync(dist2_out, d2, 8 * PL, cudaMemcpyDeviceToHost, st));
            MP_CUDA(ctx, cudaMemcpyAsync(idx_out, ix, 8 * PL, cudaMemcpyDeviceToHost, st));
        }
        MP_CUDA(ctx, cudaStreamSynchronize(st));
        collect_phases(ctx);
        return MP_OK;
    }

    // ---- FP32 re-anchored form ----------------------------------------------
    const bool guarded = precision == MP_PREC_FP32_GUARDED;
    // The guarded form reports the exact distance of the pair it chose, so its
    // error far from hazards is the FP32 selection error (two cells' drift)
    // between candidates more than kPickSpan diagonals apart: on the full c3
    // stress series (m = 1024) 8.8e-5 at K = 1024, 6.5e-5 at K = 512.  It
    // defaults to the shorter interval for the margin.
    const int64_t K = reanchor_interval(reanchor_k > 0 ? reanchor_k : (guarded ? kGuardedReanchorK : 0),
                                        kFp32R);
    rc = reserve(ctx, fp32_scratch(n, m, !o_dev, ranges.size()) + (guarded ? guard_scratch(n, m) : 0));
    if (rc) return rc;
    Carve cv{(char*)ctx->arena};
    double* Apad = cv.take<double>(n + kFp32Pad);
    int* nchg = cv.take<int>(n);
    const int64_t nblk = (n + kThreads - 1) / kThreads;
    int* tot = cv.take<int>(nblk + 1);
    double* mean = cv.take<double>(PL + kFp32Pad);
    double* norm = cv.take<double>(PL + kFp32Pad);
    float4* rowrec = cv.take<float4>(2 * (PL + kFp32Pad));
    float4* colrec = cv.take<float4>(2 * (PL + kFp32Pad));
    unsigned long long* key = cv.take<unsigned long long>(PL);
    Fp32TileParams* desc = cv.take<Fp32TileParams>(std::max<int64_t>((int64_t)ranges.size(), 1));
    unsigned long long* counter = cv.take<unsigned long long>(1);
    double* d2 = o_dev ? dist2_out : cv.take<double>(PL);
    int64_t* ix = o_dev ? idx_out : cv.take<int64_t>(PL);

    MP_CUDA(ctx, cudaMemcpyAsync(Apad, A, 8 * n, a_dev ? cudaMemcpyDeviceToDevice
                                                       : cudaMemcpyHostToDevice, st));
    mark(ctx, 0, st);
    MP_CUDA(ctx, cudaMemsetAsync(Apad + n, 0, 8 * kFp32Pad, st));
    change_flags_kernel<<<grid_for(n), kThreads, 0, st>>>(Apad, n, nchg);
    MP_LAUNCHED(ctx);
    scan_blocks_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(nchg, n, tot);
    MP_LAUNCHED(ctx);
    scan_totals_kernel<<<1, 1, 0, st>>>(tot, nblk);
    MP_LAUNCHED(ctx);
    scan_add_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(nchg, n, tot);
    MP_LAUNCHED(ctx);
    MP_CUDA(ctx, cudaMemsetAsync(mean + PL, 0, 8 * kFp32Pad, st));
    MP_CUDA(ctx, cudaMemsetAsync(norm + PL, 0, 8 * kFp32Pad, st));
    const int64_t chunk = 256;
    welford_kernel<<<grid_for((PL + chunk - 1) / chunk), kThreads, 0, st>>>(Apad, m, PL, chunk, nchg,
                                                                           mean, norm);
    MP_LAUNCHED(ctx);
    pack_fp32_kernel<<<grid_for(PL + kFp32Pad), kThreads, 0, st>>>(
        Apad, m, PL, kFp32R / 2, PL + kFp32Pad, mean, norm, rowrec, colrec);
    MP_LAUNCHED(ctx);
    const float ulim = (float)(1.0 + 1.0 / (double)m);
    init_keys_kernel<<<grid_for(PL), kThreads, 0, st>>>(
        key, PL, (unsigned long long)host_ord_f32(ulim) << 32);
    MP_LAUNCHED(ctx);
    mark(ctx, 1, st);
    if (ndiag > 0) {
        // one descriptor per diagonal range, all merging into the same keys
        std::vector<Fp32TileParams> Ps;
        int64_t ntiles = 0;
        for (const DiagRange& r : ranges) {
            Fp32TileParams Q{};
            Q.rowrec = rowrec;
            Q.colrec = colrec;
            Q.A = Apad;
            Q.mean = mean;
            Q.m = m;
            Q.PL = PL;
            Q.g_lo = r.lo;
            Q.g_hi = r.hi;
            Q.K = K;
            int64_t nt = 0;
            fp32_tile_plan(PL, r.lo, r.hi, K, kFp32R, Q.nbands, Q.seg_per_pair, nt);
            Q.tile_begin = ntiles;
            ntiles += nt;
            Q.key = key;
            Ps.push_back(Q);
        }
        Fp32TileParams& P = Ps[0];  // the guarded form has exactly one range
        if (guarded) {
            // hazard windows (prefix counts over PL + 1 entries) and FP64 terms
            int* hz = cv.take<int>(PL + 1);
            const int64_t hblk = (PL + 1 + kThreads - 1) / kThreads;
            int* htot = cv.take<int>(hblk + 1);
            double* pre = cv.take<double>(PL);
            double* suf = cv.take<double>(PL);
            double* gdf = cv.take<double>(PL);
            double* gdg = cv.take<double>(PL);
            const int64_t blk = K + 32 * kFp32R + 1;  // look back K + 32R windows
            const int64_t nb = (PL + blk - 1) / blk;
            hazard_block_minima_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(norm, PL, blk,
                                                                                  pre, suf);
            MP_LAUNCHED(ctx);
            hazard_flags_kernel<<<grid_for(PL + 1), kThreads, 0, st>>>(norm, pre, suf, PL, blk, hz);
            MP_LAUNCHED(ctx);
            scan_blocks_kernel<<<(unsigned)hblk, kThreads, 0, st>>>(hz, PL + 1, htot);
            MP_LAUNCHED(ctx);
            scan_totals_kernel<<<1, 1, 0, st>>>(htot, hblk);
            MP_LAUNCHED(ctx);
            scan_add_kernel<<<(unsigned)hblk, kThreads, 0, st>>>(hz, PL + 1, htot);
            MP_LAUNCHED(ctx);
            guard_terms_kernel<<<grid_for(PL), kThreads, 0, st>>>(Apad, m, PL, mean, gdf, gdg);
            MP_LAUNCHED(ctx);
            P.hazard = hz;
            P.norm = norm;
            P.df = gdf;
            P.dg = gdg;
        }
        MP_CUDA(ctx, cudaMemcpyAsync(desc, Ps.data(), sizeof(Fp32TileParams) * Ps.size(),
                                     cudaMemcpyHostToDevice, st));
        MP_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
        // the guarded form's keys name candidate groups, resolved in FP64 below
        launch_fp32_join<kFp32R>(desc, (int)Ps.size(), ntiles, counter, st, guarded);
        MP_LAUNCHED(ctx);
        if (guarded) {
            // the same tiles again: the FP64 pass evaluates those the FP32 pass skipped
            MP_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
            launch_fp64_guard<kFp32R>(desc, 1, ntiles, counter, st);
            MP_LAUNCHED(ctx);
            // near duplicates below the FP32 resolution floor: exact pairs among them
            int* ndl = cv.take<int>(kNearDupCap);
            int* ndc = cv.take<int>(1);
            const unsigned long long init = (unsigned long long)host_ord_f32(ulim) << 32;
            MP_CUDA(ctx, cudaMemsetAsync(ndc, 0, sizeof(int), st));
            neardup_collect_kernel<<<grid_for(PL), kThreads, 0, st>>>(key, PL, kNearDupU, init, ndl,
                                                                      ndc, kNearDupCap);
            MP_LAUNCHED(ctx);
            int nd = 0;
            MP_CUDA(ctx, cudaMemcpyAsync(&nd, ndc, sizeof(int), cudaMemcpyDeviceToHost, st));
            MP_CUDA(ctx, cudaStreamSynchronize(st));
            ctx->near_duplicates = nd;
            if (nd > 0 && nd <= kNearDupCap) {
                neardup_reset_kernel<<<grid_for(nd), kThreads, 0, st>>>(ndl, nd, key, init);
                MP_LAUNCHED(ctx);
                NearDupParams N{};
                N.A = Apad;
                N.mean = mean;
                N.norm = norm;
                N.m = m;
                N.PL = PL;
                N.g_lo = P.g_lo;
                N.g_hi = P.g_hi;
                N.list = ndl;
                N.count = nd;
                N.key = key;
                N.ulim = ulim;
                const int64_t nt = ((int64_t)nd + 31) / 32;
                neardup_pairs_kernel<<<(unsigned)(nt * nt), 256, 0, st>>>(N);
                MP_LAUNCHED(ctx);
            }
        }
        // the descriptor copy above reads host stack memory: finish it before returning
        MP_CUDA(ctx, cudaStreamSynchronize(st));
    }
    mark(ctx, 2, st);
    if (guarded)  // group keys; the chosen pair's distance from a centred FP64 dot product
        finalize_fp32_guarded_kernel<<<grid_for(PL), kThreads, 0, st>>>(
            key, PL, (double)m, Apad, mean, norm, ranges.empty() ? 0 : ranges[0].lo,
            ranges.empty() ? 0 : ranges[0].hi, d2, ix);
    else
        finalize_fp32_kernel<<<grid_for(PL), kThreads, 0, st>>>(key, PL, (double)m, Apad, mean, norm,
                                                                0, d2, ix);
    MP_LAUNCHED(ctx);
    mark(ctx, 3, st);
    if (!o_dev) {
        MP_CUDA(ctx, cudaMemcpyAsync(dist2_out, d2, 8 * PL, cudaMemcpyDeviceToHost, st));
        MP_CUDA(ctx, cudaMemcpyAsync(idx_out, ix, 8 * PL, cudaMemcpyDeviceToHost, st));
    }
    MP_CUDA(ctx, cudaStreamSynchronize(st));
    collect_phases(ctx);
    return MP_OK;
}

}  // namespace

extern "C" {

int mp_selfjoin(mp_context* ctx, const double* A, int64_t n, int64_t m, int64_t excl,
                int precision, int64_t reanchor_k, int64_t blocklen, int64_t diag_lo,
                int64_t diag_hi, double* dist2_out, int64_t* idx_out, void* stream) {
    Sizes S;
    int rc = check_join_args(ctx, A, n, m, excl, diag_lo, diag_hi, dist2_out, idx_out, S);
    if (rc) return rc;
    std::vector<DiagRange> ranges;
    if (S.hi > S.lo) ranges.push_back({S.lo, S.hi});
    return selfjoin_ranges(ctx, A, n, m, precision, reanchor_k, blocklen, S, ranges, dist2_out,
                           idx_out, stream);
}

int mp_selfjoin_ranges(mp_context* ctx, const double* A, int64_t n, int64_t m, int64_t excl,
                       int precision, int64_t reanchor_k, int64_t blocklen, const int64_t* ranges,
                       int64_t count, double* dist2_out, int64_t* idx_out, void* stream) {
    Sizes S;
    int rc = check_join_args(ctx, A, n, m, excl, 0, 0, dist2_out, idx_out, S);
    if (rc) return rc;
    if (count < 0 || (count > 0 && !ranges))
        return fail(ctx, MP_ERR_INVALID_ARG, "bad diagonal range list");
    std::vector<DiagRange> list;
    for (int64_t i = 0; i < count; ++i) {
        if (ranges[2 * i] > ranges[2 * i + 1])
            return fail(ctx, MP_ERR_INVALID_ARG, "diagonal range %lld has lo > hi", (long long)i);
        const int64_t lo = std::max(ranges[2 * i], S.lo), hi = std::min(ranges[2 * i + 1], S.hi);
        if (hi > lo) list.push_back({lo, hi});
    }
    return selfjoin_ranges(ctx, A, n, m, precision, reanchor_k, blocklen, S, list, dist2_out,
                           idx_out, stream);
}

int mp_window_stats(mp_context* ctx, const double* A, int64_t n, int64_t m, double* muS_out,
                    double* sInv_out, void* stream) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    if (!A || !muS_out || !sInv_out) return fail(ctx, MP_ERR_INVALID_ARG, "null buffer");
    if (m < 1 || n < m) return fail(ctx, MP_ERR_INVALID_ARG, "need 1 <= m <= n");
    MP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    ctx->launches = 0;
    const int64_t PL = n - m + 1;
    int rc = reserve(ctx, align_up(8 * n) * 3 + align_up(8 * PL) * 2 + 4096);
    if (rc) return rc;
    Carve cv{(char*)ctx->arena};
    double* Ad = cv.take<double>(n);
    double* cs = cv.take<double>(n);
    double* cs2 = cv.take<double>(n);
    double* mu = cv.take<double>(PL);
    double* si = cv.take<double>(PL);
    MP_CUDA(ctx, cudaMemcpyAsync(Ad, A, 8 * n, cudaMemcpyDefault, st));
    ref_prefix_kernel<<<1, kPrefixThreads, 0, st>>>(Ad, n, cs, cs2);
    MP_LAUNCHED(ctx);
    ref_stats_kernel<<<grid_for(PL), kThreads, 0, st>>>(cs, cs2, PL, m, mu, si);
    MP_LAUNCHED(ctx);
    MP_CUDA(ctx, cudaMemcpyAsync(muS_out, mu, 8 * PL, cudaMemcpyDefault, st));
    MP_CUDA(ctx, cudaMemcpyAsync(sInv_out, si, 8 * PL, cudaMemcpyDefault, st));
    MP_CUDA(ctx, cudaStreamSynchronize(st));
    return MP_OK;
}

int mp_prescrimp(mp_context* ctx, const double* A, int64_t n, int64_t m, double stride,
                 double* dist2_out, int64_t* idx_out, void* stream) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    if (!A || !dist2_out || !idx_out) return fail(ctx, MP_ERR_INVALID_ARG, "null buffer");
    if (m < 2) return fail(ctx, MP_ERR_INVALID_ARG, "window length m=%lld < 2", (long long)m);
    if (n < m)
        return fail(ctx, MP_ERR_INVALID_ARG,
                    "time series is shorter than the window length (n=%lld, m=%lld)",
                    (long long)n, (long long)m);
    const int64_t PL = n - m + 1;
    if (PL >= (1ll << 31))
        return fail(ctx, MP_ERR_NOT_SUPPORTED, "profile length %lld exceeds 2^31-1", (long long)PL);
    // ScrimpppOrig.cpp:49: stepSize = floor(prescrimp_stride * windowSize)
    const double stepf = std::floor(stride * (double)m);
    if (!(stepf >= 1.0) || stepf > (double)INT32_MAX)
        return fail(ctx, MP_ERR_INVALID_ARG, "PreSCRIMP step floor(%g * %lld) must be >= 1",
                    stride, (long long)m);
    MP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    ctx->launches = 0;
    const int64_t step = (int64_t)stepf;
    const int64_t Q = (PL + step - 1) / step;
    const MemSpace sd = mem_space(dist2_out, ctx->device), si = mem_space(idx_out, ctx->device);
    if (sd == MemSpace::OtherDevice || si == MemSpace::OtherDevice)
        return fail(ctx, MP_ERR_INVALID_ARG,
                    "dist2_out and idx_out must be host memory or device memory of the "
                    "context's device %d", ctx->device);
    const bool o_dev = sd == MemSpace::Device;
    if ((si == MemSpace::Device) != o_dev)
        return fail(ctx, MP_ERR_INVALID_ARG, "dist2_out and idx_out live in different memory spaces");
    size_t bytes = align_up(8 * (size_t)n) * 3 + align_up(8 * (size_t)PL) * 4 +
                   align_up(8 * (size_t)Q) * 2 + 4096;
    if (!o_dev) bytes += align_up(8 * (size_t)PL) * 2;
    int rc = reserve(ctx, bytes);
    if (rc) return rc;
    Carve cv{(char*)ctx->arena};
    double* Ad = cv.take<double>(n);
    double* cs = cv.take<double>(n);
    double* cs2 = cv.take<double>(n);
    double* mean = cv.take<double>(PL);
    double* sigma = cv.take<double>(PL);
    unsigned long long* kex = cv.take<unsigned long long>(PL);
    unsigned long long* kix = cv.take<unsigned long long>(PL);
    unsigned long long* rex = cv.take<unsigned long long>(Q);
    unsigned long long* rix = cv.take<unsigned long long>(Q);
    double* d2 = o_dev ? dist2_out : cv.take<double>(PL);
    int64_t* ix = o_dev ? idx_out : cv.take<int64_t>(PL);
    MP_CUDA(ctx, cudaMemcpyAsync(Ad, A, 8 * n, cudaMemcpyDefault, st));
    ref_prefix_kernel<<<1, kPrefixThreads, 0, st>>>(Ad, n, cs, cs2);
    MP_LAUNCHED(ctx);
    orig_stats_kernel<<<grid_for(PL), kThreads, 0, st>>>(cs, cs2, PL, m, mean, sigma);
    MP_LAUNCHED(ctx);
    prescrimp_keys_init_kernel<<<grid_for(PL), kThreads, 0, st>>>(kex, PL);
    MP_LAUNCHED(ctx);
    prescrimp_keys_init_kernel<<<grid_for(PL), kThreads, 0, st>>>(kix, PL);
    MP_LAUNCHED(ctx);
    prescrimp_keys_init_kernel<<<grid_for(Q), kThreads, 0, st>>>(rex, Q);
    MP_LAUNCHED(ctx);
    prescrimp_keys_init_kernel<<<grid_for(Q), kThreads, 0, st>>>(rix, Q);
    MP_LAUNCHED(ctx);
    PreScrimpParams P{};
    P.A = Ad;
    P.mean = mean;
    P.sigma = sigma;
    P.n = n;
    P.m = m;
    P.PL = PL;
    P.excl = m / 4;  // ScrimpppOrig.cpp:73
    P.step = step;
    P.Q = Q;
    P.kex = kex;
    P.kix = kix;
    P.rex = rex;
    P.rix = rix;
    P.idx_bits = bits_for((uint64_t)PL);
    launch_prescrimp(P, st);  // two kernels
    ++ctx->launches;
    MP_LAUNCHED(ctx);
    prescrimp_finalize_kernel<<<grid_for(PL), kThreads, 0, st>>>(kex, kix, PL, P.idx_bits, d2, ix);
    MP_LAUNCHED(ctx);
    if (!o_dev) {
        MP_CUDA(ctx, cudaMemcpyAsync(dist2_out, d2, 8 * PL, cudaMemcpyDeviceToHost, st));
        MP_CUDA(ctx, cudaMemcpyAsync(idx_out, ix, 8 * PL, cudaMemcpyDeviceToHost, st));
    }
    MP_CUDA(ctx, cudaStreamSynchronize(st));
    return MP_OK;
}

int mp_first_qt(mp_context* ctx, const double* A, int64_t n, int64_t m, int64_t d_lo, int64_t d_hi,
                double* qt, void* stream) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    if (!A || !qt) return fail(ctx, MP_ERR_INVALID_ARG, "null buffer");
    if (m < 1 || n < m || d_lo < 0 || d_hi > n - m + 1 || d_hi < d_lo)
        return fail(ctx, MP_ERR_INVALID_ARG, "bad diagonal range");
    MP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    ctx->launches = 0;
    const int64_t nd = d_hi - d_lo;
    int rc = reserve(ctx, align_up(8 * n) + align_up(8 * std::max<int64_t>(nd, 1)) + 4096);
    if (rc) return rc;
    Carve cv{(char*)ctx->arena};
    double* Ad = cv.take<double>(n);
    double* q = cv.take<double>(nd);
    MP_CUDA(ctx, cudaMemcpyAsync(Ad, A, 8 * n, cudaMemcpyDefault, st));
    if (nd > 0) {
        first_qt_kernel<<<grid_for(nd), kThreads, 0, st>>>(Ad, m, d_lo, d_hi, q);
        MP_LAUNCHED(ctx);
        MP_CUDA(ctx, cudaMemcpyAsync(qt, q, 8 * nd, cudaMemcpyDefault, st));
    }
    MP_CUDA(ctx, cudaStreamSynchronize(st));
    return MP_OK;
}

int mp_eval_diag_block_triangle(mp_context* ctx, double* prof_colmin, int64_t* idx_colmin,
                                double* prof_rowmin, int64_t* idx_rowmin, double* tmpQ,
                                int64_t blocklen, int64_t trianglen, const double* A_hor,
                                const double* A_vert, int64_t m, const double* s_hor,
                                const double* mu_hor, const double* s_vert, const double* mu_vert,
                                int64_t baserow, int64_t basecol, void* stream) {
    if (!ctx) return MP_ERR_INVALID_ARG;
    if (!prof_colmin || !idx_colmin || !prof_rowmin || !idx_rowmin || !tmpQ || !A_hor || !A_vert ||
        !s_hor || !mu_hor || !s_vert || !mu_vert)
        return fail(ctx, MP_ERR_INVALID_ARG, "null buffer");
    if (blocklen < 1 || trianglen < 0 || m < 1 || baserow < 0 || basecol < 0)
        return fail(ctx, MP_ERR_INVALID_ARG, "bad block geometry");
    const int64_t T = trianglen;
    if (T == 0) return MP_OK;
    if (baserow + T >= (1ll << 31) || basecol + T >= (1ll << 31))
        return fail(ctx, MP_ERR_NOT_SUPPORTED, "neighbour indices beyond 2^31");
    MP_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    ctx->launches = 0;

    // The two profile views: one region if they overlap, two otherwise.
    const ptrdiff_t dp = prof_rowmin - prof_colmin;
    const ptrdiff_t di = idx_rowmin - idx_colmin;
    const bool overlap = (dp > -(ptrdiff_t)T && dp < (ptrdiff_t)T);
    if (overlap && dp != di)
        return fail(ctx, MP_ERR_INVALID_ARG, "aliased profile views need matching index views");
    int64_t col_off, row_off, region;
    double* region_p0 = nullptr;
    int64_t* region_i0 = nullptr;
    if (overlap) {
        const int64_t lo = std::min<int64_t>(0, dp);
        col_off = -lo;
        row_off = dp - lo;
        region = std::max<int64_t>(T, dp + T) - lo;
        region_p0 = prof_colmin + lo;
        region_i0 = idx_colmin + lo;
    } else {
        col_off = 0;
        row_off = T;
        region = 2 * T;
    }
    const int64_t nrec = T + kFp64Pad;
    const int64_t nq = std::min<int64_t>(blocklen, T);
    size_t need = 2 * align_up(32 * (size_t)nrec) + 2 * align_up(8 * (size_t)nq) +
                  2 * align_up(8 * (size_t)region) * 2 + 2 * align_up(8 * (size_t)(T + m)) +
                  4 * align_up(8 * (size_t)T) + align_up(8 * (size_t)(region + kFp64ThrPad)) +
                  4096;
    int rc = reserve(ctx, need);
    if (rc) return rc;
    Carve cv{(char*)ctx->arena};
    double4* colrec = cv.take<double4>(nrec);
    double4* rowrec = cv.take<double4>(nrec);
    double* q = cv.take<double>(nq);
    double* qout = cv.take<double>(nq);
    double* prof = cv.take<double>(region);
    int64_t* pidx = cv.take<int64_t>(region);
    unsigned long long* kex = cv.take<unsigned long long>(region);
    unsigned long long* kid = cv.take<unsigned long long>(region);
    double* ah = cv.take<double>(T + m);
    double* av = cv.take<double>(T + m);
    double* sh = cv.take<double>(T);
    double* mh = cv.take<double>(T);
    double* sv = cv.take<double>(T);
    double* mv = cv.take<double>(T);
    double* thr = cv.take<double>(region + kFp64ThrPad);
    const cudaMemcpyKind K = cudaMemcpyDefault;
    MP_CUDA(ctx, cudaMemcpyAsync(ah, A_hor, 8 * (T + m), K, st));
    MP_CUDA(ctx, cudaMemcpyAsync(av, A_vert, 8 * (T + m), K, st));
    MP_CUDA(ctx, cudaMemcpyAsync(sh, s_hor, 8 * T, K, st));
    MP_CUDA(ctx, cudaMemcpyAsync(mh, mu_hor, 8 * T, K, st));
    MP_CUDA(ctx, cudaMemcpyAsync(sv, s_vert, 8 * T, K, st));
    MP_CUDA(ctx, cudaMemcpyAsync(mv, mu_vert, 8 * T, K, st));
    MP_CUDA(ctx, cudaMemcpyAsync(q, tmpQ, 8 * nq, K, st));
    if (overlap) {
        MP_CUDA(ctx, cudaMemcpyAsync(prof, region_p0, 8 * region, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(pidx, region_i0, 8 * region, K, st));
    } else {
        MP_CUDA(ctx, cudaMemcpyAsync(prof, prof_colmin, 8 * T, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(pidx, idx_colmin, 8 * T, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(prof + T, prof_rowmin, 8 * T, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(pidx + T, idx_rowmin, 8 * T, K, st));
    }
    MP_CUDA(ctx, cudaMemsetAsync(colrec + T, 0, 32 * kFp64Pad, st));
    MP_CUDA(ctx, cudaMemsetAsync(rowrec + T, 0, 32 * kFp64Pad, st));
    pack_fp64_kernel<<<grid_for(T), kThreads, 0, st>>>(ah, m, T, sh, mh, colrec);
    MP_LAUNCHED(ctx);
    pack_fp64_kernel<<<grid_for(T), kThreads, 0, st>>>(av, m, T, sv, mv, rowrec);
    MP_LAUNCHED(ctx);
    block_keys_init_kernel<<<grid_for(region), kThreads, 0, st>>>(prof, region, kex, kid);
    MP_LAUNCHED(ctx);
    init_keys_kernel<<<grid_for(region + kFp64ThrPad), kThreads, 0, st>>>(
        reinterpret_cast<unsigned long long*>(thr), region + kFp64ThrPad, no_threshold_bits());
    MP_LAUNCHED(ctx);

    Fp64BandParams P{};
    const int R = pick_fp64_R(nq);
    P.colrec = colrec;
    P.rowrec = rowrec;
    P.qt0 = q;
    P.qt_out = qout;
    P.g_lo = 0;
    P.g_hi = nq;
    P.nbands = (nq + 32 * R - 1) / (32 * R);
    P.blk_origin = 0;
    P.B = blocklen;
    P.Tbase = T;
    P.kexact = kex;
    P.kidx = kid;
    P.key_stride = region;
    P.shards = 1;
    P.row_key_off = row_off;
    P.col_key_off = col_off;
    P.row_nb_off = baserow;
    P.col_nb_off = basecol;
    P.m = (double)m;
    P.floor = -1.7976931348623157e308;
    const int ib = bits_for((uint64_t)std::max(baserow + T, basecol + T));
    P.idx_bits = ib;
    P.key_vlo = key_vlo_bits(m);
    P.thr = thr;
    P.thr_eps = fp64_threshold_eps(ib);
    P.thr_tiny = fp64_threshold_tiny(P.m);
    launch_band(R, P, st);
    MP_LAUNCHED(ctx);
    block_finalize_kernel<<<grid_for(region), kThreads, 0, st>>>(kex, kid, region, 1, region, ib,
                                                                 prof, pidx);
    MP_LAUNCHED(ctx);
    MP_CUDA(ctx, cudaMemcpyAsync(tmpQ, qout, 8 * nq, K, st));
    if (overlap) {
        MP_CUDA(ctx, cudaMemcpyAsync(region_p0, prof, 8 * region, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(region_i0, pidx, 8 * region, K, st));
    } else {
        MP_CUDA(ctx, cudaMemcpyAsync(prof_colmin, prof, 8 * T, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(idx_colmin, pidx, 8 * T, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(prof_rowmin, prof + T, 8 * T, K, st));
        MP_CUDA(ctx, cudaMemcpyAsync(idx_rowmin, pidx + T, 8 * T, K, st));
    }
    MP_CUDA(ctx, cudaStreamSynchronize(st));
    return MP_OK;
}

}  // extern "C"
