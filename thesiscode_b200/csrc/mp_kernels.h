// Kernel declarations and launch parameter blocks shared by the mpgpu
// translation units (device code and the C-ABI layer).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

struct mp_context;

namespace mpgpu {

// Memory budget of a context (0 = none); defined with the context in mp_capi.cu.
size_t ctx_budget(const mp_context* ctx);
int ctx_device(const mp_context* ctx);

// ---- preparation (mp_prep.cu) ----------------------------------------------
constexpr int kPrefixThreads = 256;  // ref_prefix_kernel: one block of this many threads
constexpr int kPrefixChunk = 1024;   // elements of A per shared-memory chunk
__global__ void ref_prefix_kernel(const double* A, int64_t n, double* cs, double* cs2);
__global__ void ref_stats_kernel(const double* cs, const double* cs2, int64_t PL, int64_t m,
                                 double* muS, double* sInv);
__global__ void first_qt_kernel(const double* A, int64_t m, int64_t d_lo, int64_t d_hi,
                                double* qt);
__global__ void pack_fp64_kernel(const double* Apad, int64_t m, int64_t count, const double* sInv,
                                 const double* muS, double4* rec);
__global__ void change_flags_kernel(const double* A, int64_t n, int* chg);
__global__ void scan_blocks_kernel(int* x, int64_t n, int* block_tot);
__global__ void scan_totals_kernel(int* tot, int64_t nblocks);
__global__ void scan_add_kernel(int* x, int64_t n, const int* tot);
__global__ void welford_kernel(const double* A, int64_t m, int64_t PL, int64_t chunk,
                               const int* nchg, double* mean_out, double* norm_out);
__global__ void pack_fp32_kernel(const double* A, int64_t m, int64_t PL, int H, int64_t count,
                                 const double* mean, const double* norm, float4* rowrec,
                                 float4* colrec);

// ---- FP64 diagonal-band join (mp_join_fp64.cu) ------------------------------
// Diagonal g (g_lo <= g < g_hi) meets column j in row r = j + g, for
// j < Tbase - g.  The reference's block geometry (blocks of B diagonals
// starting at blk_origin, triangle length T = Tbase - block start) decides
// per cell whether the fused or the separately rounded arithmetic applies.
struct Fp64BandParams {
    const double4* colrec;  // colrec[j] = {A_hor[j], A_hor[j+m], s_hor[j], mu_hor[j]}
    const double4* rowrec;  // rowrec[r] = {A_vert[r], A_vert[r+m], s_vert[r], mu_vert[r]}
    const double* qt0;      // qt0[g - g_lo]: running dot product at j = 0
    double* qt_out;         // optional: dot product after the last cell, per diagonal
    int64_t g_lo, g_hi, nbands;
    int64_t blk_origin, B, Tbase;
    unsigned long long* kexact;  // [shards][key_stride] ordered score, max-merged
    unsigned long long* kidx;    // [shards][key_stride] truncated score | neighbour
    int64_t key_stride;
    int shards;
    int64_t row_key_off, col_key_off;  // key slot of row r / column j
    int64_t row_nb_off, col_nb_off;    // neighbour written for column j / row r
    double m;
    double floor;  // only scores strictly above it are merged (-1: reference init)
    int idx_bits;
    long long key_vlo;  // bit pattern of the index key's lower range end (idx_key_f64)
    // Selection thresholds, one per key slot plus kFp64ThrPad slots of padding
    // (initialised to -DBL_MAX).  Every merge raises thr[slot] to a value a
    // little below the merged score (fp64_threshold_below); a cell whose score
    // does not exceed its row's and its column's thresholds can change neither
    // key, so a column step whose cells all fall below them skips selection.
    double* thr;
    double thr_eps;   // relative margin, wider than the index key's resolution
    double thr_tiny;  // absolute margin near v = m - score = 0
};
constexpr int kFp64WarpsPerBlock = 4;
constexpr int64_t kFp64ThrPad = 64 * 8 + 64;  // >= the 34R + R rows staged past a band's end
// Threshold stored after merging `score` (see Fp64BandParams::thr): below the
// score by more than the index key's resolution, so every cell whose index key
// could still tie or beat the key of a merged cell exceeds it.  Host-callable
// so the margin can be checked without a GPU.
__host__ __device__ inline double fp64_threshold_below(double score, double m, double eps,
                                                       double tiny) {
    const double v = m - score > 0.0 ? m - score : 0.0;
    return m - (v * (1.0 + eps) + tiny);
}
// Margins for a key with idx_bits index bits: the index key keeps 57 - idx_bits
// mantissa bits of v, i.e. a relative resolution of 2^(idx_bits - 57); eps is
// eight times that, tiny covers |v| near 0, where the key clamps.
inline double fp64_threshold_eps(int idx_bits) { return std::ldexp(1.0, idx_bits - 54); }
inline double fp64_threshold_tiny(double m) { return std::ldexp(m, -40); }
template <int R>
void launch_fp64_band(const Fp64BandParams& P, cudaStream_t s);

// ---- FP32 re-anchored tile join (mp_join_fp32.cu) ---------------------------
// One series of a (batched) join.  Its tiles are numbered
// [tile_begin, tile_begin + npairs * seg_per_pair) in the launch's tile space;
// a launch that runs only a slice of them (the request server's epochs) starts
// at the series' local tile tile_skip.
struct Fp32TileParams {
    const float4* rowrec;  // pairs (x[j], x[j+H]) of df, dg, nn; 2 float4 per row
    const float4* colrec;  // duplicated, negated column terms; 2 float4 per column
    const double* A;       // series (FP64) for the anchors
    const double* mean;    // window means (FP64)
    int64_t m, PL;
    int64_t g_lo, g_hi;    // diagonals evaluated
    int64_t K;             // columns per tile = re-anchor interval
    int64_t nbands;        // bands of 32R diagonals
    int64_t seg_per_pair;  // tiles per band pair (k, nbands-1-k), max over pairs
    int64_t tile_begin;    // first tile of this series in the launch
    int64_t tile_skip;     // local tile that launch tile tile_begin stands for (0: all)
    unsigned long long* key;  // [PL] (ordered u << 32 | neighbour or group), min-merged
    // Guarded form only (all null otherwise): hazard[w] = number of hazard
    // windows among [0, w) (PL + 1 entries); FP64 inverse norms and
    // recurrence terms for the FP64 tiles.
    const int* hazard;
    const double* norm;
    const double* df;
    const double* dg;
};
#ifdef __CUDACC__
// Local tile lt of a series -> (band, column segment): band pair p = lt /
// seg_per_pair holds bands p and nbands-1-p, whose lengths are nearly
// complementary; the pair's tiles are its first band's segments, then the
// second's.  False for the unused tail of a pair.  (Host-callable too, so the
// tile space can be checked without a GPU.)
__host__ __device__ __forceinline__ bool fp32_tile_of(const Fp32TileParams& P, int64_t lt, int64_t span,
                                             int64_t& band, int64_t& seg) {
    const int64_t p = lt / P.seg_per_pair;
    int64_t s = lt % P.seg_per_pair;
    const int64_t nseg0 = (P.PL - (P.g_lo + p * span) + P.K - 1) / P.K;
    if (s < nseg0) {
        band = p;
        seg = s;
        return true;
    }
    s -= nseg0;
    const int64_t p2 = P.nbands - 1 - p;
    if (p2 <= p) return false;
    const int64_t nseg1 = (P.PL - (P.g_lo + p2 * span) + P.K - 1) / P.K;
    band = p2;
    seg = s;
    return s < nseg1;
}
// Guarded form: does the tile (band start gb, columns [j0, j1)) touch a
// hazard window, as a column or as a row (rows j + g, g in [gb, gb + span))?
__device__ __forceinline__ bool fp32_tile_hazardous(const Fp32TileParams& P, int64_t gb, int64_t j0,
                                                    int64_t j1, int span) {
    const int64_t rs = min(j0 + gb, P.PL), re = min(j1 + gb + span, P.PL);
    return (P.hazard[j1] - P.hazard[j0]) > 0 || (P.hazard[re] - P.hazard[rs]) > 0;
}

// FP32 profile keys, min-merged: (ordered u << 32) | neighbour.  With group
// keys (the guarded form) the tile kernel finds a minimum's lane but not which
// of the lane's R diagonals holds it, so its keys name a group of adjacent
// candidate neighbours instead: bit 31 of the low word set, the group's first
// candidate in bits 0..30, and (count - 1) in the low 3 bits of the high word
// -- below the form's 2^-15 resolution of u, which keeps 0x80 in the low byte
// of u's pattern.  Keys with bit 31 clear (FP64 tiles, exact pairs, the
// initial key) name the neighbour itself.
constexpr unsigned kFp32GroupBit = 0x80000000u;
// A group key is resolved among its candidates and kPickSpan more on each
// side (FP32 ranking noise between adjacent diagonals does not stop at a
// group's edge): of the candidates q in [lo, lo + n) (n <= kPickSlots) that
// are partners of window i in the join (0 <= q < PL, g_lo <= |i - q| < g_hi),
// the one whose window has the largest centred FP64 correlation with window
// i, ties to the smaller index; NaN (flat) candidates never win; -1 when none
// qualifies.  A, mean and norm (inverse centred norms) as in the tile kernel;
// A holds at least kPickSlots - 1 values of padding past the series.  About
// kPickSlots * m FMAs.  Host-callable too, so the candidate rules can be
// checked without a GPU.
constexpr int kPickSpan = 4;
constexpr int kPickSlots = 8 + 2 * kPickSpan;
__host__ __device__ inline double pick_fma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
__host__ __device__ inline int64_t fp32_pick_neighbour(const double* A, const double* mean,
                                                       const double* norm, int64_t m, int64_t PL,
                                                       int64_t g_lo, int64_t g_hi, int64_t i,
                                                       int64_t lo, int n) {
    constexpr int W = kPickSlots;
    const int64_t hi = lo + (int64_t)n < PL ? lo + (int64_t)n : PL;
    lo = lo > 0 ? lo : 0;
    double c[W], w[W];
#pragma unroll
    for (int a = 0; a < W; ++a) c[a] = 0.0;
    const double mi = mean[i];
    double sx = 0.0;
#pragma unroll
    for (int a = 0; a < W - 1; ++a) w[a] = A[lo + a];
    int64_t t = 0;
    for (; t + W <= m; t += W) {
#pragma unroll
        for (int k = 0; k < W; ++k) {
            w[(k + W - 1) % W] = A[lo + t + k + W - 1];
            const double x = A[i + t + k] - mi;
            sx += x;
#pragma unroll
            for (int a = 0; a < W; ++a) c[a] = pick_fma(x, w[(k + a) % W], c[a]);
        }
    }
    for (; t < m; ++t) {
        const double x = A[i + t] - mi;
        sx += x;
#pragma unroll
        for (int a = 0; a < W; ++a) c[a] = pick_fma(x, A[lo + t + a], c[a]);
    }
    // sum_t x_t (A[q+t] - mean_q) = c - mean_q * sum_t x_t; the common factor
    // norm[i] > 0 does not change the ranking
    int64_t best = -1;
    double bs = -__builtin_huge_val();
#pragma unroll
    for (int a = 0; a < W; ++a) {
        const int64_t q = lo + a;
        const int64_t g = q > i ? q - i : i - q;
        if (q < hi && g >= g_lo && g < g_hi) {
            const double sc = (c[a] - mean[q] * sx) * norm[q];
            if (sc > bs) {
                bs = sc;
                best = q;
            }
        }
    }
    return best;
}
#endif
// Persistent launch over `nseries` descriptors (device array) holding `total`
// tiles; warps take tiles from *counter (zeroed by the caller beforehand).
// group: the keys name candidate groups (see kFp32GroupBit) instead of
// neighbours, which the finalisation resolves in FP64.
template <int R>
void launch_fp32_join(const Fp32TileParams* series_dev, int nseries, int64_t total,
                      unsigned long long* counter, cudaStream_t s, bool group = false);
template <int R>
void configure_fp32_join();
// Guarded form (mp_guard.cu): hazard windows and the FP64 pass over their tiles.
#ifdef __CUDACC__
// The hazard rule, host-callable so that it can be checked without a GPU.
// Window w is a hazard when it is flat (NaN inverse norm) or its inverse norm
// exceeds kGuardRatio times the smallest inverse norm among windows
// [w - (blk - 1), w]; that minimum comes from a van Herk / Gil-Werman sliding
// minimum: prefix and suffix minima within blocks of blk windows (fmin ignores
// NaN, so flat windows never lower it).
constexpr double kGuardRatio = 16.0;
// Block b: pre[i] = min nn[b*blk .. i], suf[i] = min nn[i .. end of block b].
__host__ __device__ inline void hazard_block_minima(const double* nn, int64_t PL, int64_t blk,
                                                    int64_t b, double* pre, double* suf) {
    const int64_t i0 = b * blk;
    if (i0 >= PL) return;
    const int64_t i1 = i0 + blk < PL ? i0 + blk : PL;
    double v = nn[i0];
    for (int64_t i = i0; i < i1; ++i) {
        v = fmin(v, nn[i]);
        pre[i] = v;
    }
    v = nn[i1 - 1];
    for (int64_t i = i1 - 1; i >= i0; --i) {
        v = fmin(v, nn[i]);
        suf[i] = v;
    }
}
// 1 when window w (< PL) is a hazard, from the block minima above.
__host__ __device__ inline int hazard_flag(const double* nn, const double* pre, const double* suf,
                                           int64_t blk, int64_t w) {
    const int64_t look = blk - 1;
    double mn;
    if (w < look) {
        mn = pre[w];
    } else {
        const int64_t a = w - look;
        mn = (a % blk == 0) ? pre[w] : fmin(suf[a], pre[w]);
    }
    const double x = nn[w];
    return (x != x || x > kGuardRatio * mn) ? 1 : 0;
}
#endif
__global__ void hazard_block_minima_kernel(const double* nn, int64_t PL, int64_t blk, double* pre,
                                           double* suf);
__global__ void hazard_flags_kernel(const double* nn, const double* pre, const double* suf,
                                    int64_t PL, int64_t blk, int* flag);
__global__ void guard_terms_kernel(const double* A, int64_t m, int64_t PL, const double* mean,
                                   double* df, double* dg);
// Persistent FP64 pass over the same tile space as launch_fp32_join; only
// tiles that touch a hazard window do work (counter zeroed beforehand).
template <int R>
void launch_fp64_guard(const Fp32TileParams* series_dev, int nseries, int64_t total,
                       unsigned long long* counter, cudaStream_t s);
// Near-duplicate pass of the guarded form (mp_guard.cu).
struct NearDupParams {
    const double* A;
    const double* mean;
    const double* norm;  // FP64 inverse norms (NaN: flat)
    int64_t m, PL;
    int64_t g_lo, g_hi;  // pairs on diagonals [g_lo, g_hi) only
    const int* list;     // the collected windows
    int64_t count;
    unsigned long long* key;
    float ulim;
};
__global__ void neardup_collect_kernel(const unsigned long long* key, int64_t PL, float tau,
                                       unsigned long long init, int* list, int* count, int cap);
__global__ void neardup_reset_kernel(const int* list, int count, unsigned long long* key,
                                     unsigned long long init);
__global__ void neardup_pairs_kernel(const NearDupParams P);
// Re-anchor interval K (columns per FP32 tile) from the caller's value: 1024
// when not positive, at most 2^31 (every profile is shorter, so a longer
// interval changes nothing and the rounding below cannot overflow), rounded
// up to a multiple of the R columns a chunk processes.
inline int64_t reanchor_interval(int64_t k, int R) {
    int64_t K = k > 0 ? k : 1024;
    if (K > (int64_t(1) << 31)) K = int64_t(1) << 31;
    return ((K + R - 1) / R) * R;
}
// Tile count and seg_per_pair of one series (host helper).
void fp32_tile_plan(int64_t PL, int64_t g_lo, int64_t g_hi, int64_t K, int R, int64_t& nbands,
                    int64_t& seg_per_pair, int64_t& ntiles);

// ---- PreSCRIMP (mp_prescrimp.cu) -------------------------------------------------
struct PreScrimpParams {
    const double* A;      // series, n samples
    const double* mean;   // window means (reference order)
    const double* sigma;  // window standard deviations (reference order)
    int64_t n, m, PL, excl;
    int64_t step;         // floor(stride * m): query i_t = t * step
    int64_t Q;            // number of queries
    unsigned long long* kex;  // [PL] ordered distance, min-merged
    unsigned long long* kix;  // [PL] ordered distance (high bits) | neighbour, min-merged
    unsigned long long* rex;  // [Q] a query's own best (distance)
    unsigned long long* rix;  // [Q] ... (neighbour)
    int idx_bits;
};
__global__ void orig_stats_kernel(const double* cs, const double* cs2, int64_t PL, int64_t m,
                                  double* mean, double* sigma);
__global__ void prescrimp_keys_init_kernel(unsigned long long* a, int64_t count);
__global__ void prescrimp_finalize_kernel(const unsigned long long* kex,
                                          const unsigned long long* kix, int64_t PL, int idx_bits,
                                          double* d2, int64_t* idx);
// Query rows then diagonal walks (2 launches).
void launch_prescrimp(const PreScrimpParams& P, cudaStream_t s);

// ---- finalisation (mp_finalize.cu) -------------------------------------------
__global__ void init_keys_kernel(unsigned long long* k, int64_t count, unsigned long long v);
__global__ void finalize_fp64_kernel(const unsigned long long* kexact, const unsigned long long* kidx,
                                     int64_t key_stride, int shards, int64_t PL, double m,
                                     int idx_bits, double* d2, int64_t* idx);
__global__ void finalize_fp32_kernel(const unsigned long long* key, int64_t PL, double m,
                                     const double* A, const double* mean, const double* norm,
                                     int refine, double* d2, int64_t* idx);
__global__ void finalize_fp32_guarded_kernel(const unsigned long long* key, int64_t PL, double m,
                                             const double* A, const double* mean, const double* norm,
                                             int64_t g_lo, int64_t g_hi, double* d2, int64_t* idx);
__global__ void block_keys_init_kernel(const double* prof, int64_t count, unsigned long long* kexact,
                                       unsigned long long* kidx);
__global__ void block_finalize_kernel(const unsigned long long* kexact, const unsigned long long* kidx,
                                      int64_t key_stride, int shards, int64_t count, int idx_bits,
                                      double* prof, int64_t* idx);

}  // namespace mpgpu
