// Allocation-free FP32 self-join (mp_selfjoin_fp32_noalloc).
//
// Some callers cannot allocate device memory when they need a profile: a host
// framework that owns the whole device through its own memory pool and forbids
// any other allocator, or code on a latency-critical path where a cudaMalloc
// (which can synchronise the device) is not acceptable.  mp_selfjoin cannot
// serve them, because it sizes and allocates its scratch per call.  This entry
// point runs the same FP32 re-anchored join with the same kernels, but its
// scratch is one file-scope __device__ array of fixed size: every GPU that
// loads the library holds it (MPGPU_NOALLOC_SCRATCH_BYTES, about 13 MB) until
// the process exits.  The caller passes device input and output buffers; no
// call here allocates or frees memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/mpgpu.h"
#include "mp_common.cuh"
#include "mp_kernels.h"

namespace mpgpu {
namespace {

constexpr int64_t kMaxN = MPGPU_NOALLOC_MAX_N;
constexpr int kR = 8;                   // diagonals per lane, as in mp_selfjoin
constexpr int64_t kPad = 64 * 8 + 64;   // zero padding behind the series and records
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;


// Carve-up of the scratch for a series of n samples (PL = n - m + 1 <= n).
struct Layout {
    size_t a, chg, tot, mean, norm, row, col, key, desc, counter, end;
};
constexpr Layout layout_for(int64_t n) {
    Layout L{};
    size_t o = 0;
    L.a = o;       o += align_up(8 * (size_t)(n + kPad));                         // series + padding
    L.chg = o;     o += align_up(4 * (size_t)n);                                  // change counts
    L.tot = o;     o += align_up(4 * (size_t)((n + kThreads - 1) / kThreads + 1));
    L.mean = o;    o += align_up(8 * (size_t)(n + kPad));
    L.norm = o;    o += align_up(8 * (size_t)(n + kPad));
    L.row = o;     o += align_up(32 * (size_t)(n + kPad));                        // row records
    L.col = o;     o += align_up(32 * (size_t)(n + kPad));                        // column records
    L.key = o;     o += align_up(8 * (size_t)n);                                  // profile keys
    L.desc = o;    o += align_up(sizeof(Fp32TileParams));
    L.counter = o; o += align_up(sizeof(unsigned long long));                     // tile counter
    L.end = o;
    return L;
}
constexpr size_t kScratchBytes = layout_for(kMaxN).end;
static_assert(kScratchBytes <= MPGPU_NOALLOC_SCRATCH_BYTES,
              "MPGPU_NOALLOC_SCRATCH_BYTES must cover the layout at MPGPU_NOALLOC_MAX_N");

// The scratch.  Host code must not pass `g_noalloc_scratch` to a kernel: on the
// host the name is a stand-in, not a device address.  Its device address comes
// from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MPGPU_NOALLOC_SCRATCH_BYTES];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};  // per device ordinal, set by the first call there

int report(char* err, size_t len, int status, const char* fmt, ...) {
    if (err && len) {
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(err, len, fmt, ap);
        va_end(ap);
    }
    return status;
}

// Device address of the scratch on the current device; the first call on a
// device looks it up (and sets the join kernel's shared-memory limit there).
// Both are kept for the life of the process: after a cudaDeviceReset of that
// device they are stale, so a reset is not supported once a call has run.
int setup_current_device(void** out, int* dev_out, char* err, size_t len) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return report(err, len, MP_ERR_NO_DEVICE, "no current CUDA device");
    }
    if (dev >= kMaxDevices)
        return report(err, len, MP_ERR_NOT_SUPPORTED, "device ordinal %d >= %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
            major < 10) {
            cudaGetLastError();
            return report(err, len, MP_ERR_NO_DEVICE, "device %d is not an sm_100 device", dev);
        }
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return report(err, len, MP_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
                          cudaGetErrorString(e));
        }
        configure_fp32_join<kR>();
        if (cudaGetLastError() != cudaSuccess)
            return report(err, len, MP_ERR_CUDA, "configuring the join kernel failed");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    *dev_out = dev;
    return MP_OK;
}


// Writes the tile descriptor from a kernel argument, so that nothing on the
// stream reads host memory after this function has returned.
__global__ void noalloc_desc_kernel(Fp32TileParams* d, Fp32TileParams P) { *d = P; }

}  // namespace
}  // namespace mpgpu

using namespace mpgpu;

extern "C" int mp_selfjoin_fp32_noalloc(const double* A_dev, int64_t n, int64_t m, int64_t excl,
                                        int64_t reanchor_k, double* dist2_dev, int64_t* idx_dev,
                                        void* stream, char* err, size_t err_len) {
    if (err && err_len) err[0] = '\0';
    if (!A_dev || !dist2_dev || !idx_dev)
        return report(err, err_len, MP_ERR_INVALID_ARG, "null buffer");
    if (m < 2)
        return report(err, err_len, MP_ERR_INVALID_ARG, "window length m=%lld < 2", (long long)m);
    if (n < m)
        return report(err, err_len, MP_ERR_INVALID_ARG,
                      "time series is shorter than the window length (n=%lld, m=%lld)",
                      (long long)n, (long long)m);
    if (n > kMaxN)
        return report(err, err_len, MP_ERR_NOT_SUPPORTED,
                      "n=%lld exceeds the allocation-free limit of %lld samples "
                      "(use mp_selfjoin for longer series)",
                      (long long)n, (long long)kMaxN);
    void* base = nullptr;
    int dev = -1;
    int rc = setup_current_device(&base, &dev, err, err_len);
    if (rc != MP_OK) return rc;
    if (mem_space(A_dev, dev) != MemSpace::Device || mem_space(dist2_dev, dev) != MemSpace::Device ||
        mem_space(idx_dev, dev) != MemSpace::Device)
        return report(err, err_len, MP_ERR_INVALID_ARG,
                      "A, dist2 and idx must be device memory of the current device %d", dev);

    cudaStream_t st = (cudaStream_t)stream;
    const Layout L = layout_for(n);
    char* b = static_cast<char*>(base);
    double* Apad = reinterpret_cast<double*>(b + L.a);
    int* nchg = reinterpret_cast<int*>(b + L.chg);
    int* tot = reinterpret_cast<int*>(b + L.tot);
    double* mean = reinterpret_cast<double*>(b + L.mean);
    double* norm = reinterpret_cast<double*>(b + L.norm);
    float4* rowrec = reinterpret_cast<float4*>(b + L.row);
    float4* colrec = reinterpret_cast<float4*>(b + L.col);
    unsigned long long* key = reinterpret_cast<unsigned long long*>(b + L.key);
    Fp32TileParams* desc = reinterpret_cast<Fp32TileParams*>(b + L.desc);
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(b + L.counter);

    const int64_t PL = n - m + 1, nblk = (n + kThreads - 1) / kThreads;
    const int64_t ex = excl < 0 ? m / 4 : excl;
    const int64_t lo = ex + 1, hi = PL;
    const int64_t K = reanchor_interval(reanchor_k, kR);

    // The scratch keeps whatever the previous call left in it.  Every region
    // read below is first written on this stream: the series copy and its
    // zero padding, the change counts and scan totals, the statistics and
    // their zero padding, both record arrays (padding included), the keys
    // (set to the "no neighbour" key), the descriptor and the tile counter,
    // which must start at zero.
    cudaMemcpyAsync(Apad, A_dev, 8 * n, cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(Apad + n, 0, 8 * kPad, st);
    change_flags_kernel<<<grid_for(n), kThreads, 0, st>>>(Apad, n, nchg);
    scan_blocks_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(nchg, n, tot);
    scan_totals_kernel<<<1, 1, 0, st>>>(tot, nblk);
    scan_add_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(nchg, n, tot);
    cudaMemsetAsync(mean + PL, 0, 8 * kPad, st);
    cudaMemsetAsync(norm + PL, 0, 8 * kPad, st);
    const int64_t chunk = 256;
    welford_kernel<<<grid_for((PL + chunk - 1) / chunk), kThreads, 0, st>>>(Apad, m, PL, chunk, nchg,
                                                                           mean, norm);
    pack_fp32_kernel<<<grid_for(PL + kPad), kThreads, 0, st>>>(Apad, m, PL, kR / 2, PL + kPad, mean,
                                                               norm, rowrec, colrec);
    const float ulim = (float)(1.0 + 1.0 / (double)m);
    init_keys_kernel<<<grid_for(PL), kThreads, 0, st>>>(key, PL,
                                                        (unsigned long long)host_ord_f32(ulim) << 32);
    if (hi > lo) {
        Fp32TileParams P{};
        P.rowrec = rowrec;
        P.colrec = colrec;
        P.A = Apad;
        P.mean = mean;
        P.m = m;
        P.PL = PL;
        P.g_lo = lo;
        P.g_hi = hi;
        P.K = K;
        int64_t ntiles = 0;
        fp32_tile_plan(PL, lo, hi, K, kR, P.nbands, P.seg_per_pair, ntiles);
        P.tile_begin = 0;
        P.key = key;
        noalloc_desc_kernel<<<1, 1, 0, st>>>(desc, P);
        cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st);
        launch_fp32_join<kR>(desc, 1, ntiles, counter, st);
    }
    finalize_fp32_kernel<<<grid_for(PL), kThreads, 0, st>>>(key, PL, (double)m, Apad, mean, norm, 0,
                                                            dist2_dev, idx_dev);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return report(err, err_len, MP_ERR_CUDA, "launch failed: %s", cudaGetErrorString(e));
    return MP_OK;
}
