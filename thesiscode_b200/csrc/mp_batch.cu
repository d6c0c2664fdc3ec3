// Batched self-joins: many series of uneven length and window size solved by
// one persistent join launch (the FP32 re-anchored tile kernel walking a tile
// space that spans every series), with the preparation and finalisation of all
// series batched into single launches.  The whole device sequence is captured
// once into a CUDA graph and replayed for every run of the plan.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mpgpu.h"
#include "mp_common.cuh"
#include "mp_kernels.h"
#include "mp_prep_device.cuh"

namespace mpgpu {
namespace {

constexpr int kR = 8;
constexpr int64_t kPad = 64 * 8 + 64;  // elements/records past each series' end

struct BatchSeries {
    int64_t n, m, PL;
    int64_t in_off;   // input staging (elements)
    int64_t a_off;    // padded FP64 series and change counts (n + kPad)
    int64_t w_off;    // mean / norm (PL + kPad)
    int64_t r_off;    // row and column records (PL + kPad records, 2 float4 each)
    int64_t k_off;    // keys and outputs (PL)
};

// One block row per series (blockIdx.y), grid-stride over its elements.
#define FOR_SERIES_ELEMS(count) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (count); i += (int64_t)gridDim.x * blockDim.x)

__global__ void batch_convert_kernel(const BatchSeries* __restrict__ S, const void* __restrict__ in,
                                     int input_f32, double* __restrict__ A) {
    const BatchSeries s = S[blockIdx.y];
    FOR_SERIES_ELEMS(s.n + kPad) {
        double v = 0.0;
        if (i < s.n)
            v = input_f32 ? (double)reinterpret_cast<const float*>(in)[s.in_off + i]
                          : reinterpret_cast<const double*>(in)[s.in_off + i];
        A[s.a_off + i] = v;
    }
}

// Per-series inclusive count of value changes (one block per series; the
// block walks the series in blockDim-sized pieces carrying the running sum).
__global__ void batch_change_count_kernel(const BatchSeries* __restrict__ S,
                                          const double* __restrict__ A, int* __restrict__ nchg) {
    __shared__ int wsum[32];
    __shared__ int carry;
    const BatchSeries s = S[blockIdx.x];
    const double* a = A + s.a_off;
    int* out = nchg + s.a_off;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t base = 0; base < s.n; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        int v = (i > 0 && i < s.n && a[i] != a[i - 1]) ? 1 : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(kFullMask, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) wsum[w] = v;
        __syncthreads();
        if (w == 0) {
            int t = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(kFullMask, t, o);
                if (lane >= o) t += u;
            }
            wsum[lane] = t;
        }
        __syncthreads();
        if (w > 0) v += wsum[w - 1];
        v += carry;
        if (i < s.n) out[i] = v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = v;
        __syncthreads();
    }
}

__global__ void batch_welford_kernel(const BatchSeries* __restrict__ S, const double* __restrict__ A,
                                     const int* __restrict__ nchg, int64_t chunk,
                                     double* __restrict__ mean, double* __restrict__ norm) {
    const BatchSeries s = S[blockIdx.y];
    const int64_t nchunks = (s.PL + chunk - 1) / chunk;
    FOR_SERIES_ELEMS(nchunks) {
        welford_chunk(A + s.a_off, s.m, s.PL, chunk, i, nchg + s.a_off, mean + s.w_off,
                      norm + s.w_off);
    }
    FOR_SERIES_ELEMS(kPad) {
        mean[s.w_off + s.PL + i] = 0.0;
        norm[s.w_off + s.PL + i] = 0.0;
    }
}

__global__ void batch_pack_kernel(const BatchSeries* __restrict__ S, const double* __restrict__ A,
                                  const double* __restrict__ mean, const double* __restrict__ norm,
                                  float4* __restrict__ rowrec, float4* __restrict__ colrec,
                                  unsigned long long* __restrict__ key, const unsigned* __restrict__ ulim_key) {
    const BatchSeries s = S[blockIdx.y];
    FOR_SERIES_ELEMS(s.PL + kPad) {
        pack_fp32_record(A + s.a_off, s.m, s.PL, kR / 2, mean + s.w_off, norm + s.w_off, i,
                         rowrec + 2 * s.r_off, colrec + 2 * s.r_off);
        if (i < s.PL) key[s.k_off + i] = (unsigned long long)ulim_key[blockIdx.y] << 32;
    }
}

__global__ void batch_finalize_kernel(const BatchSeries* __restrict__ S,
                                      const unsigned long long* __restrict__ key,
                                      double* __restrict__ d2, int64_t* __restrict__ idx) {
    const BatchSeries s = S[blockIdx.y];
    const float ulim = (float)(1.0 + 1.0 / (double)s.m);
    const unsigned long long init = (unsigned long long)ord_f32(ulim) << 32;
    FOR_SERIES_ELEMS(s.PL) {
        const unsigned long long k = key[s.k_off + i];
        if (k >= init) {
            d2[s.k_off + i] = 2.0 * s.m + 2.0;
            idx[s.k_off + i] = 0;
        } else {
            d2[s.k_off + i] = 2.0 * s.m * (double)unord_f32((unsigned)(k >> 32));
            idx[s.k_off + i] = (int64_t)(k & 0xffffffffull);
        }
    }
}


}  // namespace
}  // namespace mpgpu

using namespace mpgpu;

struct mp_batch {
    int device = 0;
    int input_f32 = 0;
    int64_t count = 0;
    std::vector<BatchSeries> series;
    std::vector<Fp32TileParams> tiles;
    int64_t total_tiles = 0;
    double cells = 0;
    int64_t in_elems = 0, a_elems = 0, w_elems = 0, r_recs = 0, k_elems = 0;
    int64_t launches = 0;
    char* dev = nullptr;  // one device allocation, carved
    size_t dev_bytes = 0;
    void* in_stage = nullptr;  // pinned host staging (input)
    char* out_stage = nullptr;  // pinned host staging (d2 then idx)
    // device pointers
    BatchSeries* d_series = nullptr;
    Fp32TileParams* d_tiles = nullptr;
    unsigned* d_ulim = nullptr;
    unsigned long long* d_counter = nullptr;
    void* d_in = nullptr;
    double* d_A = nullptr;
    int* d_nchg = nullptr;
    double* d_mean = nullptr;
    double* d_norm = nullptr;
    float4* d_row = nullptr;
    float4* d_col = nullptr;
    unsigned long long* d_key = nullptr;
    double* d_d2 = nullptr;
    int64_t* d_idx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string err;
};

namespace {

// Host copies between the caller's per-series arrays and the pinned staging
// buffers run on several threads: one thread moves a few GB/s, and the
// staging copies of a large batch are gigabytes.
template <class F>
void for_series_parallel(int64_t count, F body) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int64_t nt = std::min<int64_t>(std::min<unsigned>(hw, 16u), std::max<int64_t>(count, 1));
    if (nt <= 1) {
        for (int64_t s = 0; s < count; ++s) body(s);
        return;
    }
    std::vector<std::thread> pool;
    for (int64_t t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            for (int64_t s = t; s < count; s += nt) body(s);
        });
    for (auto& th : pool) th.join();
}


int enqueue_batch(mp_batch* b, cudaStream_t st) {
    const int maxy = (int)std::min<int64_t>(b->count, 65535);
    if (b->count > 65535) return MP_ERR_NOT_SUPPORTED;
    const dim3 grid(64, maxy);
    batch_convert_kernel<<<grid, 256, 0, st>>>(b->d_series, b->d_in, b->input_f32, b->d_A);
    batch_change_count_kernel<<<(unsigned)b->count, 256, 0, st>>>(b->d_series, b->d_A, b->d_nchg);
    batch_welford_kernel<<<grid, 256, 0, st>>>(b->d_series, b->d_A, b->d_nchg, 256, b->d_mean,
                                               b->d_norm);
    batch_pack_kernel<<<grid, 256, 0, st>>>(b->d_series, b->d_A, b->d_mean, b->d_norm, b->d_row,
                                            b->d_col, b->d_key, b->d_ulim);
    cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long), st);
    launch_fp32_join<kR>(b->d_tiles, (int)b->count, b->total_tiles, b->d_counter, st);
    batch_finalize_kernel<<<grid, 256, 0, st>>>(b->d_series, b->d_key, b->d_d2, b->d_idx);
    b->launches = 6;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        b->err = cudaGetErrorString(e);
        return MP_ERR_CUDA;
    }
    return MP_OK;
}


}  // namespace

extern "C" {

int mp_batch_create(mp_context* ctx, int64_t count, const int64_t* lengths, const int64_t* windows,
                    const int64_t* reanchor_k, int input_type, mp_batch** out) {
    if (!ctx || !out || !lengths || !windows || count < 1) return MP_ERR_INVALID_ARG;
    if (input_type != 0 && input_type != 1) return MP_ERR_INVALID_ARG;
    if (count > 65535) return MP_ERR_NOT_SUPPORTED;
    *out = nullptr;
    // the batch lives on the context's device, whatever the caller's current one
    const int dev = ctx_device(ctx);
    if (cudaSetDevice(dev) != cudaSuccess) {
        cudaGetLastError();
        return MP_ERR_NO_DEVICE;
    }
    mp_batch* b = new mp_batch();
    b->device = dev;
    b->input_f32 = input_type;
    b->count = count;
    int64_t in = 0, a = 0, w = 0, r = 0, k = 0, tiles = 0;
    for (int64_t s = 0; s < count; ++s) {
        const int64_t n = lengths[s], m = windows[s];
        if (m < 2 || n < m || n - m + 1 >= (1ll << 31)) {
            delete b;
            return MP_ERR_INVALID_ARG;
        }
        BatchSeries bs{};
        bs.n = n;
        bs.m = m;
        bs.PL = n - m + 1;
        bs.in_off = in;
        bs.a_off = a;
        bs.w_off = w;
        bs.r_off = r;
        bs.k_off = k;
        in += n;
        a += n + kPad;
        w += bs.PL + kPad;
        r += bs.PL + kPad;
        k += bs.PL;
        b->series.push_back(bs);
        Fp32TileParams P{};
        P.m = m;
        P.PL = bs.PL;
        P.g_lo = m / 4 + 1;
        P.g_hi = bs.PL;
        P.K = reanchor_interval(reanchor_k ? reanchor_k[s] : 0, kR);
        int64_t nt = 0;
        fp32_tile_plan(bs.PL, P.g_lo, P.g_hi, P.K, kR, P.nbands, P.seg_per_pair, nt);
        if (P.g_hi <= P.g_lo) nt = 0;
        P.tile_begin = tiles;
        tiles += nt;
        b->tiles.push_back(P);
        const double L = (double)std::max<int64_t>(bs.PL - m / 4 - 1, 0);
        b->cells += L * (L + 1) / 2;
    }
    b->in_elems = in;
    b->a_elems = a;
    b->w_elems = w;
    b->r_recs = r;
    b->k_elems = k;
    b->total_tiles = tiles;
    const size_t esz = input_type ? 4 : 8;
    size_t bytes = align_up(sizeof(BatchSeries) * count) + align_up(sizeof(Fp32TileParams) * count) +
                   align_up(4 * count) + align_up(8) + align_up(esz * in) + align_up(8 * a) + align_up(4 * a) + 2 * align_up(8 * w) +
                   2 * align_up(32 * r) + align_up(8 * k) + align_up(8 * k) + align_up(8 * k);
    if (ctx_budget(ctx) && bytes > ctx_budget(ctx)) {
        delete b;
        return MP_ERR_BUDGET;
    }
    if (cudaMalloc((void**)&b->dev, bytes) != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return MP_ERR_OUT_OF_MEMORY;
    }
    b->dev_bytes = bytes;
    char* p = b->dev;
    auto take = [&](size_t n) {
        char* q = p;
        p += align_up(n);
        return q;
    };
    b->d_series = (BatchSeries*)take(sizeof(BatchSeries) * count);
    b->d_tiles = (Fp32TileParams*)take(sizeof(Fp32TileParams) * count);
    b->d_ulim = (unsigned*)take(4 * count);
    b->d_counter = (unsigned long long*)take(8);
    b->d_in = take(esz * in);
    b->d_A = (double*)take(8 * a);
    b->d_nchg = (int*)take(4 * a);
    b->d_mean = (double*)take(8 * w);
    b->d_norm = (double*)take(8 * w);
    b->d_row = (float4*)take(32 * r);
    b->d_col = (float4*)take(32 * r);
    b->d_key = (unsigned long long*)take(8 * k);
    b->d_d2 = (double*)take(8 * k);
    b->d_idx = (int64_t*)take(8 * k);
    std::vector<unsigned> ulim(count);
    for (int64_t s = 0; s < count; ++s) {
        Fp32TileParams& P = b->tiles[s];
        const BatchSeries& bs = b->series[s];
        P.rowrec = b->d_row + 2 * bs.r_off;
        P.colrec = b->d_col + 2 * bs.r_off;
        P.A = b->d_A + bs.a_off;
        P.mean = b->d_mean + bs.w_off;
        P.key = b->d_key + bs.k_off;
        ulim[s] = host_ord_f32((float)(1.0 + 1.0 / (double)bs.m));
    }
    if (cudaMemcpy(b->d_series, b->series.data(), sizeof(BatchSeries) * count,
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_tiles, b->tiles.data(), sizeof(Fp32TileParams) * count,
                   cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_ulim, ulim.data(), 4 * count, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(b->dev);
        delete b;
        return MP_ERR_CUDA;
    }
    configure_fp32_join<kR>();
    *out = b;
    return MP_OK;
}

int mp_batch_destroy(mp_batch* b) {
    if (!b) return MP_ERR_INVALID_ARG;
    cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->dev) cudaFree(b->dev);
    if (b->in_stage) cudaFreeHost(b->in_stage);
    if (b->out_stage) cudaFreeHost(b->out_stage);
    delete b;
    return MP_OK;
}

double mp_batch_cells(const mp_batch* b) { return b ? b->cells : 0.0; }
int64_t mp_batch_tiles(const mp_batch* b) { return b ? b->total_tiles : 0; }
int64_t mp_batch_launch_count(const mp_batch* b) { return b ? b->launches : 0; }

int mp_batch_upload(mp_batch* b, const void* const* series, void* stream) {
    if (!b || !series) return MP_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MP_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t esz = b->input_f32 ? 4 : 8;
    if (!b->in_stage && cudaHostAlloc(&b->in_stage, esz * b->in_elems, 0) != cudaSuccess) {
        cudaGetLastError();
        b->in_stage = nullptr;
        return MP_ERR_OUT_OF_MEMORY;
    }
    cudaStreamSynchronize(st);  // the staging buffer may still feed a previous copy
    for_series_parallel(b->count, [&](int64_t s) {
        std::memcpy((char*)b->in_stage + esz * b->series[s].in_off, series[s], esz * b->series[s].n);
    });
    if (cudaMemcpyAsync(b->d_in, b->in_stage, esz * b->in_elems, cudaMemcpyHostToDevice, st) !=
        cudaSuccess)
        return MP_ERR_CUDA;
    return MP_OK;
}

int mp_batch_launch(mp_batch* b, void* stream) {
    if (!b) return MP_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MP_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->exec) {
        cudaStream_t cap = st;
        bool own = false;
        if (cap == nullptr) {  // the legacy stream cannot be captured
            if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess)
                return MP_ERR_CUDA;
            own = true;
        }
        if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            if (own) cudaStreamDestroy(cap);
            return MP_ERR_CUDA;
        }
        int rc = enqueue_batch(b, cap);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(cap, &g);
        if (own) cudaStreamDestroy(cap);
        if (rc != MP_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != MP_OK ? rc : MP_ERR_CUDA;
        }
        if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            cudaGetLastError();
            return MP_ERR_CUDA;
        }
        b->graph = g;
    }
    if (cudaGraphLaunch(b->exec, st) != cudaSuccess) return MP_ERR_CUDA;
    return MP_OK;
}

int mp_batch_download(mp_batch* b, double* const* dist2_out, int64_t* const* idx_out, void* stream) {
    if (!b || !dist2_out || !idx_out) return MP_ERR_INVALID_ARG;
    if (cudaSetDevice(b->device) != cudaSuccess) return MP_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->out_stage && cudaHostAlloc((void**)&b->out_stage, 16 * b->k_elems, 0) != cudaSuccess) {
        cudaGetLastError();
        b->out_stage = nullptr;
        return MP_ERR_OUT_OF_MEMORY;
    }
    if (cudaMemcpyAsync(b->out_stage, b->d_d2, 8 * b->k_elems, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaMemcpyAsync(b->out_stage + 8 * b->k_elems, b->d_idx, 8 * b->k_elems,
                        cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return MP_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return MP_ERR_CUDA;
    const double* d2 = (const double*)b->out_stage;
    const int64_t* ix = (const int64_t*)(b->out_stage + 8 * b->k_elems);
    for_series_parallel(b->count, [&](int64_t s) {
        const BatchSeries& bs = b->series[s];
        if (dist2_out[s]) std::memcpy(dist2_out[s], d2 + bs.k_off, 8 * bs.PL);
        if (idx_out[s]) std::memcpy(idx_out[s], ix + bs.k_off, 8 * bs.PL);
    });
    return MP_OK;
}

int mp_batch_run(mp_batch* b, const void* const* series, double* const* dist2_out,
                 int64_t* const* idx_out, void* stream) {
    int rc = mp_batch_upload(b, series, stream);
    if (rc) return rc;
    rc = mp_batch_launch(b, stream);
    if (rc) return rc;
    return mp_batch_download(b, dist2_out, idx_out, stream);
}

}  // extern "C"
