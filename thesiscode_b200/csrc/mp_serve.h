// Device side of the request server's epoch engine (mp_serve.cu), called by
// the host scheduler in host/mp_server.cpp.
//
// A request's FP32 re-anchored self-join is a set of independent tiles (each
// re-anchors itself in FP64), so the server runs many requests as epochs: one
// persistent launch of the FP32 tile kernel over a bounded slice of tiles
// drawn from every admitted request.  Requests that arrive meanwhile join the
// next epoch.  A request's result is the same whichever epochs its tiles land
// in (every merge is an exact 64-bit min), i.e. the same as mp_selfjoin's.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

struct mp_context;

namespace mpgpu {

// Lends ctx the device buffer `scratch` (bytes long) as its scratch for the
// calls that follow: the context neither uses nor grows its own arena, and a
// call that needs more than `bytes` fails with MP_ERR_BUDGET.  scratch =
// nullptr gives the context its own arena back.  The request server's
// workers lend each request a buffer from the server's pool, so that their
// scratch is counted in its budget and released without a device-wide
// synchronisation (mp_capi.cu).
void ctx_lend_scratch(mp_context* ctx, void* scratch, size_t bytes);

// One admitted request on the device.  All buffers come from the server's
// stream-ordered memory pool.
struct ServeJob {
    int64_t n = 0, m = 0, PL = 0;
    int64_t K = 0;                        // re-anchor interval (columns per tile)
    int64_t g_lo = 0, g_hi = 0;           // diagonals evaluated
    int64_t nbands = 0, seg_per_pair = 0;
    int64_t ntiles = 0;                   // local tiles [0, ntiles)
    int64_t next_tile = 0;                // first tile not yet launched
    double cells = 0.0;
    void* scratch = nullptr;              // series, statistics, records, keys
    size_t scratch_bytes = 0;
    double* d2 = nullptr;                 // results, resident until collected
    int64_t* idx = nullptr;
    // carved from scratch
    double* A = nullptr;
    double* mean = nullptr;
    double* norm = nullptr;
    float4* rowrec = nullptr;
    float4* colrec = nullptr;
    unsigned long long* key = nullptr;
};

// A slice of one job's tiles in an epoch.
struct ServeSlice {
    ServeJob* job;
    int64_t first, count;
};

// Device bytes of a request (scratch + resident result).
size_t serve_scratch_bytes(int64_t n, int64_t m);
size_t serve_result_bytes(int64_t n, int64_t m);

// Allocates the job's buffers from `pool` on `st`, copies the host series in
// and runs the preparation (change counts, Welford statistics, records, key
// initialisation).  Fills the tile plan.  Returns a cudaError_t.
cudaError_t serve_prepare(ServeJob& job, const double* series, int64_t n, int64_t m,
                          int64_t reanchor_k, cudaMemPool_t pool, cudaStream_t st);

// Per-epoch device state: descriptor buffers and the tile counter.
struct ServeEpochBuffers {
    static constexpr int kRing = 3;   // epochs whose descriptors may be in use
    int max_slices = 0;
    void* desc_dev[kRing] = {};       // Fp32TileParams[max_slices]
    void* desc_host[kRing] = {};      // pinned staging
    unsigned long long* counter = nullptr;
};
cudaError_t serve_epoch_buffers_create(ServeEpochBuffers& b, int max_slices);
void serve_epoch_buffers_destroy(ServeEpochBuffers& b);

// Launches one epoch (descriptor upload, counter reset, the persistent FP32
// tile kernel) on `st`, using descriptor buffer `ring_slot`.  Returns the
// launch's tile count, or -1 on a CUDA error.
int64_t serve_launch_epoch(ServeEpochBuffers& b, int ring_slot, const std::vector<ServeSlice>& slices,
                           cudaStream_t st);

// Squared distances and indices of a job whose tiles have all been launched
// (enqueued after its last epoch), then its scratch goes back to the pool.
cudaError_t serve_finalize(ServeJob& job, cudaStream_t st);

// Returns the job's remaining buffers to the pool.
void serve_release_result(ServeJob& job, cudaStream_t st);

}  // namespace mpgpu
