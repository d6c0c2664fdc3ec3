/*
 * mpgpu -- B200 (sm_100a) matrix-profile self-join, C ABI.
 *
 * Plain C types only: pointers, sizes and status codes.  Every function
 * returns MP_OK (0) or a positive mp_status; no C++ exception crosses this
 * boundary.  Buffers stay owned by the caller; the library owns its device
 * scratch through an mp_context.  One context per host thread.
 *
 * Semantics follow the reference's diagonal-blocked SCRIMP path
 * (4rchangel/ThesisCode, scrimppp/):
 *   - windows i in [0, PL), PL = n - m + 1; exclusion zone |i-j| <= excl,
 *     excl defaults to m/4 (ScrimpVertBlocked.cpp:97);
 *   - profile value = squared z-normalised distance 2m - 2*score
 *     (ScrimpVertBlocked.cpp:171-174), index = nearest neighbour window;
 *   - a window no pair improves keeps score -1 (d2 = 2m+2) and index 0
 *     (ScrimpVertBlocked.cpp:103-104); a window of exactly zero variance
 *     makes every score it touches NaN, so it never wins and is never chosen.
 */
#ifndef MPGPU_H
#define MPGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MP_OK = 0,
    MP_ERR_INVALID_ARG = 1,   /* n < m, m < 2, bad range, null pointer ... */
    MP_ERR_OUT_OF_MEMORY = 2, /* device allocation failed */
    MP_ERR_BUDGET = 3,        /* request exceeds the context's memory budget */
    MP_ERR_CUDA = 4,          /* a CUDA call failed; see mp_last_error() */
    MP_ERR_NOT_SUPPORTED = 5, /* size or option outside what is implemented */
    MP_ERR_NO_DEVICE = 6,     /* no usable sm_100 device */
    MP_ERR_IO = 7             /* a series or profile file could not be read or written */
} mp_status;

typedef enum {
    /* Operation-for-operation replica of the reference arithmetic in FP64:
     * same window statistics, same first dot products, same fused /
     * separately rounded per-cell steps as the reference's AVX2 kernel.
     * Profile values are bit-identical to the reference compiled with IEEE
     * semantics; indices agree except between candidates whose squared
     * distances tie to within ~1.2e-10 relative (n <= 2^24), where the
     * smaller neighbour index is kept. */
    MP_PREC_FP64 = 0,
    /* FP32 covariance recurrence re-anchored every reanchor_k steps by an FP64
     * dot product; window means/norms in FP64 (Welford). */
    MP_PREC_FP32_REANCHOR = 1,
    /* MP_PREC_FP32_REANCHOR plus three FP64 safeguards for ill-conditioned
     * data: tiles touching a window that is flat or has a norm over 16 times
     * smaller than the largest norm among the reanchor_k + 256 windows before
     * it (level steps, values beside constant stretches) run the recurrence
     * in FP64; windows whose best FP32 distance is below the FP32 resolution
     * floor (u = d^2/2m < 1e-3, near-duplicates) are recomputed pairwise in
     * FP64; and every window's chosen pair gets its distance from a centred
     * FP64 dot product.  On a plain random walk only the last step runs. */
    MP_PREC_FP32_GUARDED = 2
} mp_precision;

typedef struct mp_context mp_context;

/* device: CUDA ordinal.  mem_budget_bytes: ceiling for the context's device
 * scratch (0 = no ceiling); a call that would exceed it fails with
 * MP_ERR_BUDGET before allocating. */
int mp_context_create(int device, size_t mem_budget_bytes, mp_context** out);
int mp_context_destroy(mp_context* ctx);
/* Text of the last error recorded on ctx (never NULL). */
const char* mp_last_error(const mp_context* ctx);
const char* mp_status_string(int status);
/* Device bytes one self-join of (n, m, precision) needs in ctx's scratch. */
size_t mp_selfjoin_scratch_bytes(int64_t n, int64_t m, int precision);

/*
 * Whole self-join (replaces ScrimpVertBlocked::compute_matrix_profile,
 * scrimppp/src/ScrimpVertBlocked.cpp:89-195, minus the file I/O).
 *
 *   A            n doubles, host or device memory (detected).
 *   excl         exclusion zone; < 0 selects m/4.
 *   precision    mp_precision.
 *   reanchor_k   FP32 forms: columns between FP64 re-anchors (0 = 1024 for
 *                MP_PREC_FP32_REANCHOR, 512 for MP_PREC_FP32_GUARDED).
 *   blocklen     FP64 form: the reference's --blocklen (0 = 500); it decides
 *                which cells the reference evaluates with fused operations,
 *                so it is needed for bit-identical values.
 *   diag_lo/hi   evaluate diagonals [diag_lo, diag_hi) only (0,0 = all,
 *                i.e. excl+1 .. PL-1); used for sharding and for sampling.
 *   dist2_out    PL doubles: squared distances (host or device).
 *   idx_out      PL int64 neighbour indices (host or device).
 *   stream       cudaStream_t (NULL = legacy default stream).
 * The call returns after the results are written (it synchronises stream).
 * Device buffers must belong to the context's device: device memory of
 * another GPU returns MP_ERR_INVALID_ARG before anything is launched.
 */
int mp_selfjoin(mp_context* ctx, const double* A, int64_t n, int64_t m, int64_t excl,
                int precision, int64_t reanchor_k, int64_t blocklen, int64_t diag_lo,
                int64_t diag_hi, double* dist2_out, int64_t* idx_out, void* stream);

/*
 * mp_selfjoin over several diagonal ranges at once: ranges[2i], ranges[2i+1]
 * are the bounds [lo, hi) of range i (clipped to excl+1 .. PL-1; empty ones are
 * skipped).  One preparation, every range joined into the same profile, one
 * finalisation and one synchronisation -- the per-rank part of a join sharded
 * by the reference's scrimp_triv_par rule, where rank r of P evaluates
 * partitions r and 2P-1-r (scrimppp/src/ScrimpTrivialPar.cpp:200-224).  The
 * guarded form takes one range only (MP_ERR_NOT_SUPPORTED otherwise).
 */
int mp_selfjoin_ranges(mp_context* ctx, const double* A, int64_t n, int64_t m, int64_t excl,
                       int precision, int64_t reanchor_k, int64_t blocklen, const int64_t* ranges,
                       int64_t count, double* dist2_out, int64_t* idx_out, void* stream);

/*
 * One block of diagonals, the reference's kernel interface
 * (scrimppp/inc/kernels.h:7-24, scrimppp/src/kernels.cpp:368-410), evaluated
 * on the GPU in FP64 with the reference's per-cell arithmetic.  Arguments have
 * the reference's meaning: a triangle of `blocklen` adjacent diagonals and
 * `trianglen` columns; column j meets rows i = j + delta, delta < blocklen,
 * i < trianglen; scores (not distances) are max-merged with strict '>' into
 * prof_colmin[j]/idx_colmin[j] (neighbour i + baserow) and
 * prof_rowmin[i]/idx_rowmin[i] (neighbour j + basecol); tmpQ[delta] carries
 * the running dot product in and out.  The two profile views may alias one
 * array (self-join) or be disjoint (tiles).  Host or device pointers; all in
 * the same memory space.  Synchronous on stream.
 */
int mp_eval_diag_block_triangle(mp_context* ctx, double* prof_colmin, int64_t* idx_colmin,
                                double* prof_rowmin, int64_t* idx_rowmin, double* tmpQ,
                                int64_t blocklen, int64_t trianglen, const double* A_hor,
                                const double* A_vert, int64_t m, const double* s_hor,
                                const double* mu_hor, const double* s_vert, const double* mu_vert,
                                int64_t baserow, int64_t basecol, void* stream);

/* Window statistics of the reference (ScrimpSequOpt.cpp:33-79), bit-identical:
 * muS[i] = mean*sInv*sqrt(m), sInv[i] = 1/sqrt(var), i < PL. */
int mp_window_stats(mp_context* ctx, const double* A, int64_t n, int64_t m, double* muS,
                    double* sInv, void* stream);

/* First dot products of diagonals [d_lo, d_hi) (ScrimpSequOpt.cpp:81-96),
 * bit-identical: qt[d - d_lo] = sum_k A[k+d]*A[k] summed in k order. */
int mp_first_qt(mp_context* ctx, const double* A, int64_t n, int64_t m, int64_t d_lo,
                int64_t d_hi, double* qt, void* stream);

/* Kernel launches the last call on ctx made (for launch accounting). */
int64_t mp_last_launch_count(const mp_context* ctx);
/* MP_PREC_FP32_GUARDED: windows whose best FP32 distance was below the FP32
 * resolution floor (u = d^2/2m < 1e-3) and were recomputed pairwise in FP64 by
 * the last mp_selfjoin on ctx (at most 131072; -1 for other forms). */
int64_t mp_last_near_duplicates(const mp_context* ctx);

/* Phase timing: with on != 0, mp_selfjoin records CUDA events on its stream
 * around its three phases (preparation, join kernel, finalisation);
 * mp_last_phase_ms reads them after the call (milliseconds, -1 if unset). */
int mp_set_phase_timing(mp_context* ctx, int on);
int mp_last_phase_ms(const mp_context* ctx, double* prep_ms, double* join_ms,
                     double* finalize_ms);

/*
 * Batched self-joins (no counterpart in the reference: its variants join one
 * series per process).  A plan fixes `count` series (lengths, windows, FP32
 * re-anchor interval per series -- NULL = 1024 each -- and input type 0 = double,
 * 1 = float); all of them are solved by one persistent FP32 re-anchored join
 * launch, with the preparation and finalisation batched into single launches,
 * recorded once as a CUDA graph and replayed by every mp_batch_launch.
 * Results follow mp_selfjoin's conventions.  count <= 65535.
 *   mp_batch_upload    copies the caller's host series into the plan (pinned staging)
 *   mp_batch_launch    runs the captured graph on stream (asynchronous)
 *   mp_batch_download  copies the profiles to the caller's host arrays (synchronous)
 *   mp_batch_run       the three in order
 */
typedef struct mp_batch mp_batch;
int mp_batch_create(mp_context* ctx, int64_t count, const int64_t* lengths, const int64_t* windows,
                    const int64_t* reanchor_k, int input_type, mp_batch** out);
int mp_batch_destroy(mp_batch* b);
double mp_batch_cells(const mp_batch* b);
int64_t mp_batch_tiles(const mp_batch* b);
int64_t mp_batch_launch_count(const mp_batch* b);
int mp_batch_upload(mp_batch* b, const void* const* series, void* stream);
int mp_batch_launch(mp_batch* b, void* stream);
int mp_batch_download(mp_batch* b, double* const* dist2_out, int64_t* const* idx_out, void* stream);
int mp_batch_run(mp_batch* b, const void* const* series, double* const* dist2_out,
                 int64_t* const* idx_out, void* stream);

/*
 * Request server (no counterpart in the reference).  Continuous batching of
 * independent self-joins: requests are admitted while fewer than `slots` are
 * admitted and the device memory they need (scratch + resident result) fits
 * in mem_budget_bytes, the waiting request with the fewest cells first (a
 * request that has waited 2 s goes before any other, so none starves).  A finished profile stays on the
 * device until mp_server_collect copies it out (and frees it).  A request
 * larger than the whole budget is rejected (MP_ERR_BUDGET).
 *   MP_PREC_FP32_REANCHOR  one scheduler runs every admitted request as part
 *                          of epochs: one persistent launch of the FP32 tile
 *                          kernel over a bounded slice of tiles from each
 *                          (a minimum share each, the rest to the requests
 *                          with the least work left); new requests join the
 *                          next epoch.  Device memory comes from a pool of
 *                          the server's own (stream-ordered, kept between
 *                          requests, bounded by the budget).  Results equal
 *                          mp_selfjoin's with the same reanchor_k.
 *   MP_PREC_FP64, MP_PREC_FP32_GUARDED
 *                          `slots` worker threads run whole mp_selfjoin calls,
 *                          each on its own stream.
 *   mp_server_submit   copies the host series, returns a ticket, never blocks
 *   mp_server_poll     1 when finished (status set), 0 while pending
 *   mp_server_collect  waits for the ticket, copies d2/idx (may be NULL), frees;
 *                      latency = submission to finish, queue = submission to start
 */
typedef struct mp_server mp_server;
int mp_server_create(int device, size_t mem_budget_bytes, int slots, int precision,
                     int64_t reanchor_k, mp_server** out);
int mp_server_submit(mp_server* s, const double* A, int64_t n, int64_t m, int64_t* ticket);
int mp_server_poll(mp_server* s, int64_t ticket, int* status);
int mp_server_collect(mp_server* s, int64_t ticket, double* dist2_out, int64_t* idx_out,
                      double* latency_s, double* queue_s);
int mp_server_stats(mp_server* s, int64_t* completed, int64_t* rejected, int64_t* waiting,
                    int64_t* running, double* cells, size_t* bytes_in_use);
int mp_server_destroy(mp_server* s);

/*
 * Allocation-free FP32 self-join.  No counterpart in the reference (which
 * allocates its buffers per run); added for callers that must not allocate
 * device memory: a host framework that owns the whole GPU through its own
 * memory pool and forbids other allocators, or a latency-critical path where
 * cudaMalloc/cudaFree (which can synchronise the device) are not allowed.
 *
 * Same arithmetic, kernels and results as mp_selfjoin with
 * MP_PREC_FP32_REANCHOR over all diagonals, but its scratch is a fixed
 * device array of MPGPU_NOALLOC_SCRATCH_BYTES that every GPU loading this
 * library holds until the process exits, so n is limited to
 * MPGPU_NOALLOC_MAX_N samples; longer series return MP_ERR_NOT_SUPPORTED.
 * No call allocates or frees memory.
 *
 *   A_dev        n doubles in device memory of the current device.
 *   excl         exclusion zone; < 0 selects m/4.
 *   reanchor_k   columns between FP64 re-anchors (0 = 1024).
 *   dist2_dev    PL = n - m + 1 doubles (device): squared distances.
 *   idx_dev      PL int64 (device): neighbour indices.
 *   stream       cudaStream_t (NULL = legacy default stream).  The call only
 *                enqueues work: results are ready when the stream reaches
 *                this point, and A_dev must stay valid until then.
 *   err/err_len  optional buffer for a one-line error message (may be NULL).
 *
 * The first call on a device (the current device at the time of the call)
 * looks up the scratch's device address and configures the join kernel
 * there; make that first call before any stream capture.  Both are kept for
 * the life of the process, so resetting that device (cudaDeviceReset) after
 * the first call is not supported.  Buffers on another GPU are refused with
 * MP_ERR_INVALID_ARG before anything is launched.  All calls on a
 * device share the one scratch array: calls whose work overlaps on the GPU
 * (other streams, other host threads) race and corrupt each other's results,
 * so serialise them (one stream, or events between streams).
 */
#define MPGPU_NOALLOC_MAX_N 131072
#define MPGPU_NOALLOC_SCRATCH_BYTES (14u << 20)
int mp_selfjoin_fp32_noalloc(const double* A_dev, int64_t n, int64_t m, int64_t excl,
                             int64_t reanchor_k, double* dist2_dev, int64_t* idx_dev,
                             void* stream, char* err, size_t err_len);

/*
 * PreSCRIMP, the anytime front end of SCRIMP++ (replaces the PreSCRIMP phase
 * of ScrimpppOrig::compute_matrix_profile, scrimppp/src/ScrimpppOrig.cpp:
 * 130-266).  Query windows i = 0, s, 2s, ... with s = floor(stride * m) get
 * their whole distance profile (windows j with |j - i| < m/4 excluded, as in
 * the reference); every evaluated cell lowers both windows' entries; then each
 * query's best diagonal is walked s - 1 cells forward and backward.  The
 * result is an approximate profile (an upper bound of the exact one) in
 * squared distances, with the reference's initial values (+inf, index 0) for
 * windows no cell reached.  The reference convolves with FFTW; the GPU forms
 * each query cell as a direct FP64 dot product, so values agree with the
 * reference to rounding, not bit for bit, and every update is a min-merge
 * (independent of the reference's shuffled query order).
 *   A            n doubles, host or device memory.
 *   stride       the reference's --prescrimp-stride (an integer there; fractions
 *                are accepted here), s = floor(stride * m) >= 1.
 *   dist2_out    PL doubles, idx_out PL int64 (host or device, same space).
 * Synchronous on stream.
 */
int mp_prescrimp(mp_context* ctx, const double* A, int64_t n, int64_t m, double stride,
                 double* dist2_out, int64_t* idx_out, void* stream);

/* FMA throughput of this device's CUDA-core pipes in FLOP/s (2 per FMA),
 * measured with independent FMA chains: which = 0 FP32 (FFMA), 1 FP32 (f32x2
 * FFMA2), 2 FP64 (DFMA).  The join kernels' compute roofline uses it. */
int mp_measure_fma_peak(int device, int which, double* flops_per_s);

/*
 * Algorithm registry (the reference's MatProfImplFactory,
 * scrimppp/src/MatProfAlgo.cpp:11-37, exposed to C callers).
 * mp_list_algorithms writes the space-separated registered names into buf and
 * returns the length needed including the terminator.
 * mp_run_algorithm runs one registered variant end to end on files, like the
 * reference's main (scrimppp/src/main.cpp:47-80): filetype 1 = ASCII,
 * 2 = binary; blocklen/reanchor_k <= 0 keep the defaults (500 / 1024).
 * Returns MP_ERR_INVALID_ARG for an unknown name or bad parameters,
 * MP_ERR_IO when the input cannot be read (checked before any device is
 * used) or the output cannot be written, and otherwise the status of the
 * failing library call (MP_ERR_NO_DEVICE without a B200, ...).
 */
int mp_list_algorithms(char* buf, size_t len);
int mp_run_algorithm(const char* algo, const char* input_file, const char* output_file,
                     int window_length, int prescrimp_stride, int blocklen, int filetype,
                     int64_t reanchor_k, int device);

#ifdef __cplusplus
}
#endif

#endif /* MPGPU_H */
