// Device side of the request server's epoch engine (see mp_serve.h).
//
// Preparation is the FP32 form's own (the same kernels and launch shapes as
// mp_selfjoin with MP_PREC_FP32_REANCHOR); an epoch is one launch of the
// persistent FP32 tile kernel over a list of (request, first tile, tile count)
// slices; finalisation turns a request's merged keys into squared distances
// and indices.  Every allocation is stream-ordered from the server's pool, so
// nothing here waits for the device.
#include <algorithm>
#include <cstring>

#include "mp_common.cuh"
#include "mp_kernels.h"
#include "mp_serve.h"

namespace mpgpu {

namespace {

constexpr int kR = 8;                  // diagonals per lane, as in mp_selfjoin
constexpr int64_t kPad = 64 * 8 + 64;  // zero padding behind the series and records
constexpr int kThreads = 256;

struct Layout {
    size_t a, chg, tot, mean, norm, row, col, key, end;
};
Layout layout_for(int64_t n, int64_t m) {
    const int64_t PL = n - m + 1, nblk = (n + kThreads - 1) / kThreads;
    Layout L{};
    size_t o = 0;
    L.a = o;    o += align_up(8 * (size_t)(n + kPad));
    L.chg = o;  o += align_up(4 * (size_t)n);
    L.tot = o;  o += align_up(4 * (size_t)(nblk + 1));
    L.mean = o; o += align_up(8 * (size_t)(PL + kPad));
    L.norm = o; o += align_up(8 * (size_t)(PL + kPad));
    L.row = o;  o += align_up(32 * (size_t)(PL + kPad));
    L.col = o;  o += align_up(32 * (size_t)(PL + kPad));
    L.key = o;  o += align_up(8 * (size_t)PL);
    L.end = o;
    return L;
}

}  // namespace

size_t serve_scratch_bytes(int64_t n, int64_t m) { return layout_for(n, m).end; }
size_t serve_result_bytes(int64_t n, int64_t m) { return 2 * align_up(8 * (size_t)(n - m + 1)); }

cudaError_t serve_prepare(ServeJob& job, const double* series, int64_t n, int64_t m,
                          int64_t reanchor_k, cudaMemPool_t pool, cudaStream_t st) {
    const int64_t PL = n - m + 1;
    const Layout L = layout_for(n, m);
    job.n = n;
    job.m = m;
    job.PL = PL;
    job.scratch_bytes = L.end;
    cudaError_t e = cudaMallocFromPoolAsync(&job.scratch, L.end, pool, st);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync((void**)&job.d2, 8 * (size_t)PL, pool, st);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync((void**)&job.idx, 8 * (size_t)PL, pool, st);
    if (e != cudaSuccess) return e;
    char* b = static_cast<char*>(job.scratch);
    job.A = reinterpret_cast<double*>(b + L.a);
    int* nchg = reinterpret_cast<int*>(b + L.chg);
    int* tot = reinterpret_cast<int*>(b + L.tot);
    job.mean = reinterpret_cast<double*>(b + L.mean);
    job.norm = reinterpret_cast<double*>(b + L.norm);
    job.rowrec = reinterpret_cast<float4*>(b + L.row);
    job.colrec = reinterpret_cast<float4*>(b + L.col);
    job.key = reinterpret_cast<unsigned long long*>(b + L.key);

    const int64_t nblk = (n + kThreads - 1) / kThreads;
    if ((e = cudaMemcpyAsync(job.A, series, 8 * n, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(job.A + n, 0, 8 * kPad, st)) != cudaSuccess) return e;
    change_flags_kernel<<<grid_for(n), kThreads, 0, st>>>(job.A, n, nchg);
    scan_blocks_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(nchg, n, tot);
    scan_totals_kernel<<<1, 1, 0, st>>>(tot, nblk);
    scan_add_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(nchg, n, tot);
    if ((e = cudaMemsetAsync(job.mean + PL, 0, 8 * kPad, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(job.norm + PL, 0, 8 * kPad, st)) != cudaSuccess) return e;
    const int64_t chunk = 256;
    welford_kernel<<<grid_for((PL + chunk - 1) / chunk), kThreads, 0, st>>>(job.A, m, PL, chunk, nchg,
                                                                           job.mean, job.norm);
    pack_fp32_kernel<<<grid_for(PL + kPad), kThreads, 0, st>>>(job.A, m, PL, kR / 2, PL + kPad,
                                                               job.mean, job.norm, job.rowrec,
                                                               job.colrec);
    const float ulim = (float)(1.0 + 1.0 / (double)m);
    init_keys_kernel<<<grid_for(PL), kThreads, 0, st>>>(
        job.key, PL, (unsigned long long)host_ord_f32(ulim) << 32);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;

    job.K = reanchor_interval(reanchor_k, kR);
    job.g_lo = m / 4 + 1;
    job.g_hi = PL;
    job.ntiles = 0;
    job.nbands = job.seg_per_pair = 0;
    if (job.g_hi > job.g_lo)
        fp32_tile_plan(PL, job.g_lo, job.g_hi, job.K, kR, job.nbands, job.seg_per_pair, job.ntiles);
    job.next_tile = 0;
    const double c = (double)std::max<int64_t>(PL - job.g_lo, 0);
    job.cells = c * (c + 1) / 2;
    return cudaSuccess;
}

cudaError_t serve_epoch_buffers_create(ServeEpochBuffers& b, int max_slices) {
    b.max_slices = max_slices;
    const size_t bytes = sizeof(Fp32TileParams) * (size_t)max_slices;
    cudaError_t e;
    for (int i = 0; i < ServeEpochBuffers::kRing; ++i) {
        if ((e = cudaMalloc(&b.desc_dev[i], bytes)) != cudaSuccess) return e;
        if ((e = cudaMallocHost(&b.desc_host[i], bytes)) != cudaSuccess) return e;
    }
    return cudaMalloc((void**)&b.counter, sizeof(unsigned long long));
}

void serve_epoch_buffers_destroy(ServeEpochBuffers& b) {
    for (int i = 0; i < ServeEpochBuffers::kRing; ++i) {
        if (b.desc_dev[i]) cudaFree(b.desc_dev[i]);
        if (b.desc_host[i]) cudaFreeHost(b.desc_host[i]);
        b.desc_dev[i] = b.desc_host[i] = nullptr;
    }
    if (b.counter) cudaFree(b.counter);
    b.counter = nullptr;
}

int64_t serve_launch_epoch(ServeEpochBuffers& b, int ring_slot, const std::vector<ServeSlice>& slices,
                           cudaStream_t st) {
    if (slices.empty() || (int)slices.size() > b.max_slices) return -1;
    Fp32TileParams* h = static_cast<Fp32TileParams*>(b.desc_host[ring_slot]);
    int64_t total = 0;
    for (size_t i = 0; i < slices.size(); ++i) {
        const ServeJob& j = *slices[i].job;
        Fp32TileParams P{};
        P.rowrec = j.rowrec;
        P.colrec = j.colrec;
        P.A = j.A;
        P.mean = j.mean;
        P.m = j.m;
        P.PL = j.PL;
        P.g_lo = j.g_lo;
        P.g_hi = j.g_hi;
        P.K = j.K;
        P.nbands = j.nbands;
        P.seg_per_pair = j.seg_per_pair;
        P.tile_begin = total;
        P.tile_skip = slices[i].first;
        P.key = j.key;
        h[i] = P;
        total += slices[i].count;
    }
    const size_t bytes = sizeof(Fp32TileParams) * slices.size();
    if (cudaMemcpyAsync(b.desc_dev[ring_slot], h, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(b.counter, 0, sizeof(unsigned long long), st) != cudaSuccess)
        return -1;
    launch_fp32_join<kR>(static_cast<const Fp32TileParams*>(b.desc_dev[ring_slot]),
                         (int)slices.size(), total, b.counter, st);
    return cudaGetLastError() == cudaSuccess ? total : -1;
}

cudaError_t serve_finalize(ServeJob& job, cudaStream_t st) {
    finalize_fp32_kernel<<<grid_for(job.PL), kThreads, 0, st>>>(job.key, job.PL, (double)job.m, job.A,
                                                                job.mean, job.norm, 0, job.d2, job.idx);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaFreeAsync(job.scratch, st);
    job.scratch = nullptr;
    return e;
}

void serve_release_result(ServeJob& job, cudaStream_t st) {
    if (job.scratch) cudaFreeAsync(job.scratch, st);
    if (job.d2) cudaFreeAsync(job.d2, st);
    if (job.idx) cudaFreeAsync(job.idx, st);
    job.scratch = nullptr;
    job.d2 = nullptr;
    job.idx = nullptr;
}

}  // namespace mpgpu
