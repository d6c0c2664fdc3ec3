// FP64 diagonal-band join: the reference's SCRIMP recurrence evaluated with
// the reference's own per-cell arithmetic, one warp per band of 32*R
// adjacent diagonals.
//
// Reference: eval_diag_block_triangle, AVX2 branch
// (scrimppp/src/kernels.cpp:170-307), driven over blocks of blocklen
// diagonals by ScrimpVertBlocked (scrimppp/src/ScrimpVertBlocked.cpp:139-168).
// Per cell (column j, diagonal g, row r = j + g):
//   4-wide part : score = fma(QT, s_r*s_j, -(mu_j*mu_r))
//                 QT    = fma(-A[r], A[j], fma(A[r+m], A[j+m], QT))
//   remainder   : score = QT*(s_r*s_j) - mu_r*mu_j, QT = (QT + A[r+m]*A[j+m]) - A[r]*A[j]
// (every product and sum separately rounded).  A cell is in the remainder
// iff its offset in the reference block, delta, is >= 4*floor(cnt/4) with
// cnt = min(blocklen, T - j); for a diagonal that is only its last
// 3 - delta%4 cells (or all of it when delta >= blocklen & ~3).
//
// Work layout (B200): lane l of a warp owns diagonals g0 + a, a < R,
// g0 = band start + l*R; all lanes walk the same column j.  Per step a lane
// evaluates R cells: the column maximum over the warp comes from two warp
// reductions (high, then low word of the ordered score), the row maxima
// accumulate in registers for R steps and then pass through a per-warp shared
// memory ring (one writer per slot per chunk, no atomics) until the warp's
// lowest lane has seen the row.  Finished rows and columns go to global
// memory as 64-bit max reductions into one of several key shards.  One
// resident wave of warps walks the bands in a snake order (band b to warp
// b mod W in even rounds, W-1 - b mod W in odd ones), so every warp's bands
// add up to nearly the same length -- the reference's triv_par balance rule
// (ScrimpTrivialPar.cpp:200-224) carried over any number of rounds.
//
// Selection thresholds: every merge also raises a per-entry threshold to a
// value just below the merged score (fp64_threshold_below: the margin is wider
// than the index key's resolution).  A lane's row partials start at their
// rows' thresholds, and in the branch-free chunks each column step first
// evaluates its cells and compares them with their row partials and with the
// column's threshold; only when some cell of the warp exceeds one does the
// step run the (score, index) selection.  A cell that exceeds neither can
// raise neither key of its row or column (its score is below a score already
// merged there, by more than the index key resolves), so the result is the
// same as selecting every cell.  Thresholds are read as they stand (a stale
// one is only a lower bound), so the arithmetic and the keys -- and therefore
// the output -- do not depend on timing.
#include <float.h>

#include <algorithm>
#include <atomic>

#include "mp_common.cuh"
#include "mp_kernels.h"

namespace mpgpu {

namespace {

// A 32-byte record of the warp's shared-memory ring (16-byte aligned halves).
__device__ __forceinline__ double4 ring_rec(const char* p) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 16);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Which parts of a column step need the selection, voted over the warp: bit 0
// when some lane has a cell above its row partial, bit 1 when some cell is
// above the column's threshold.  Chains of predicated compares per lane
// (setp ... .or; with R = 8 two chains of 4 per test, interleaved, so the
// dependent compares are half as deep) and two votes; NaN compares false, so
// NaN cells never select.
template <int R>
__device__ __forceinline__ unsigned step_hits(const double (&sc)[R], const double (&acc)[2 * R - 1],
                                              int b, double tc) {
    bool row = false, col = false;
#pragma unroll
    for (int a = 0; a < R; ++a) {
        row |= sc[a] > acc[b + a];
        col |= sc[a] > tc;
    }
    return (__any_sync(kFullMask, row) ? 1u : 0u) | (__any_sync(kFullMask, col) ? 2u : 0u);
}
template <>
__device__ __forceinline__ unsigned step_hits<4>(const double (&sc)[4], const double (&acc)[7],
                                                 int b, double tc) {
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred pr, pc, qr, qc;\n\t"
        "setp.gt.f64 pr, %1, %5;\n\t"
        "setp.gt.or.f64 pr, %2, %6, pr;\n\t"
        "setp.gt.or.f64 pr, %3, %7, pr;\n\t"
        "setp.gt.or.f64 pr, %4, %8, pr;\n\t"
        "setp.gt.f64 pc, %1, %9;\n\t"
        "setp.gt.or.f64 pc, %2, %9, pc;\n\t"
        "setp.gt.or.f64 pc, %3, %9, pc;\n\t"
        "setp.gt.or.f64 pc, %4, %9, pc;\n\t"
        "vote.sync.any.pred qr, pr, 0xffffffff;\n\t"
        "vote.sync.any.pred qc, pc, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, qr;\n\t"
        "@qc or.b32 %0, %0, 2;\n\t"
        "}"
        : "=r"(r)
        : "d"(sc[0]), "d"(sc[1]), "d"(sc[2]), "d"(sc[3]), "d"(acc[b]), "d"(acc[b + 1]),
          "d"(acc[b + 2]), "d"(acc[b + 3]), "d"(tc));
    return r;
}
template <>
__device__ __forceinline__ unsigned step_hits<8>(const double (&sc)[8], const double (&acc)[15],
                                                 int b, double tc) {
    unsigned r;
    asm volatile(
        "{\n\t.reg .pred pr, pc, pr2, pc2, qr, qc;\n\t"
        "setp.gt.f64 pr, %1, %9;\n\t"
        "setp.gt.f64 pr2, %5, %13;\n\t"
        "setp.gt.f64 pc, %1, %17;\n\t"
        "setp.gt.f64 pc2, %5, %17;\n\t"
        "setp.gt.or.f64 pr, %2, %10, pr;\n\t"
        "setp.gt.or.f64 pr2, %6, %14, pr2;\n\t"
        "setp.gt.or.f64 pc, %2, %17, pc;\n\t"
        "setp.gt.or.f64 pc2, %6, %17, pc2;\n\t"
        "setp.gt.or.f64 pr, %3, %11, pr;\n\t"
        "setp.gt.or.f64 pr2, %7, %15, pr2;\n\t"
        "setp.gt.or.f64 pc, %3, %17, pc;\n\t"
        "setp.gt.or.f64 pc2, %7, %17, pc2;\n\t"
        "setp.gt.or.f64 pr, %4, %12, pr;\n\t"
        "setp.gt.or.f64 pr2, %8, %16, pr2;\n\t"
        "setp.gt.or.f64 pc, %4, %17, pc;\n\t"
        "setp.gt.or.f64 pc2, %8, %17, pc2;\n\t"
        "or.pred pr, pr, pr2;\n\t"
        "or.pred pc, pc, pc2;\n\t"
        "vote.sync.any.pred qr, pr, 0xffffffff;\n\t"
        "vote.sync.any.pred qc, pc, 0xffffffff;\n\t"
        "selp.u32 %0, 1, 0, qr;\n\t"
        "@qc or.b32 %0, %0, 2;\n\t"
        "}"
        : "=r"(r)
        : "d"(sc[0]), "d"(sc[1]), "d"(sc[2]), "d"(sc[3]), "d"(sc[4]), "d"(sc[5]), "d"(sc[6]),
          "d"(sc[7]), "d"(acc[b]), "d"(acc[b + 1]), "d"(acc[b + 2]), "d"(acc[b + 3]),
          "d"(acc[b + 4]), "d"(acc[b + 5]), "d"(acc[b + 6]), "d"(acc[b + 7]), "d"(tc));
    return r;
}

// Asynchronous copies global -> shared (both addresses aligned to the size):
// 16 bytes through L2 only, 8 bytes through L1.
__device__ __forceinline__ void cp_async16(char* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

// A threshold as it stands (other warps raise it with atomics meanwhile; any
// value it has held is a valid lower bound).
__device__ __forceinline__ double ld_thr(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}

__device__ __forceinline__ void flush_fp64(const Fp64BandParams& P, int shard, int64_t slot,
                                           double score, int64_t neighbour) {
    unsigned long long* ke = P.kexact + (int64_t)shard * P.key_stride + slot;
    unsigned long long* ki = P.kidx + (int64_t)shard * P.key_stride + slot;
    atomicMax(ke, ord_f64(score));
    atomicMax(ki, idx_key_f64(score, P.m, (unsigned long long)neighbour, P.idx_bits, P.key_vlo));
    // thresholds only ever hold non-negative values above their -DBL_MAX
    // start, where the signed 64-bit pattern orders like the double
    const double t = fp64_threshold_below(score, P.m, P.thr_eps, P.thr_tiny);
    if (t >= 0.0) atomicMax(reinterpret_cast<long long*>(P.thr + slot), __double_as_longlong(t));
}

// Per-warp ring of row thresholds in shared memory, indexed like the record
// ring (row t of the band at slot t % kRecRing), one double of padding after
// every 8 so that lanes reading rows 8 apart hit distinct banks.  Slots
// kRecRing .. kRecRing + kThrMirror - 1 mirror slots 0 .. kThrMirror - 1, so
// the 16 consecutive rows a lane starts in one chunk never wrap: with R = 8
// their offsets are one base plus compile-time constants.
constexpr int kThrMirror = 16;
constexpr int kThrRingDoubles = (kRecRing + kThrMirror) + (kRecRing + kThrMirror) / 8;
__device__ __forceinline__ int thr_pos(int s) { return s + (s >> 3); }
__device__ __forceinline__ int thr_off(int t) { return thr_pos(t % kRecRing); }
__device__ __forceinline__ void thr_store(double* tring, int t, double v) {
    const int s = t % kRecRing;
    tring[thr_pos(s)] = v;
    if (s < kThrMirror) tring[thr_pos(s + kRecRing)] = v;
}

// The (score, index) selection of one column step: row partials (strict '>',
// the reference's rule; a partial started at its row's threshold has no
// source (RowSrc) until a cell beats it), then the column's best cell over
// the warp from two REDUX instructions (high, then low word of the ordered
// score); the lowest winning lane parks (score, row) in the warp's column slot
// with a predicated store, so no divergent branch splits consecutive steps.
// Where a lane's 2R - 1 row partials came from: the diagonal offset a < R of
// the selected cell, as nibble k = a + 1, or 0 while partial k is still its
// row's threshold (no candidate yet).  One 64-bit register pair instead of
// 2R - 1 registers.
struct RowSrc {
    unsigned long long w;
    __device__ __forceinline__ int get(int k) const { return (int)((w >> (4 * k)) & 15ull) - 1; }
    __device__ __forceinline__ void set(int k, int a) {
        w = (w & ~(15ull << (4 * k))) | ((unsigned long long)(a + 1) << (4 * k));
    }
};
template <int R>
__device__ __forceinline__ void select_rows(int b, const double (&sc)[R], double (&acc_s)[2 * R - 1],
                                            RowSrc& acc_a) {
    static_assert(2 * R - 1 <= 16, "2R - 1 nibbles fit 64 bits");
#pragma unroll
    for (int a = 0; a < R; ++a) {
        if (sc[a] > acc_s[b + a]) {
            acc_s[b + a] = sc[a];
            acc_a.set(b + a, a);
        }
    }
}
template <int R>
__device__ __forceinline__ void select_column(const Fp64BandParams& P, int b, const double (&sc)[R],
                                              int64_t g0, int lane, double* cslot_s, int* cslot_r) {
    // lane's best cell of the column: pairwise tree, left wins ties.  A NaN
    // cell (a constant window) never selects under the reference's '>'; as
    // -DBL_MAX it also cannot hide the cell it is paired with in the tree.
    double cb[R];
    int ca[R];
#pragma unroll
    for (int a = 0; a < R; ++a) {
        cb[a] = sc[a] == sc[a] ? sc[a] : -DBL_MAX;
        ca[a] = a;
    }
#pragma unroll
    for (int w = 1; w < R; w *= 2)
#pragma unroll
        for (int a = 0; a + w < R; a += 2 * w)
            if (cb[a + w] > cb[a]) {
                cb[a] = cb[a + w];
                ca[a] = ca[a + w];
            }
    const double cbest = cb[0];
    const unsigned long long key = (cbest > P.floor) ? ord_f64(cbest) : 0ull;
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(kFullMask, hi);
    const unsigned mlo = __reduce_max_sync(kFullMask, hi == mhi ? lo : 0u);
    const bool top = (hi == mhi) && (lo == mlo) && (mhi != 0u);
    const unsigned tops = __ballot_sync(kFullMask, top);
    if (top && (tops & ((1u << lane) - 1u)) == 0u) {
        cslot_s[b] = cbest;
        cslot_r[b] = (int)(b + g0 + ca[0]);  // row - jc (rows < 2^31)
    }
}
template <int R>
__device__ __forceinline__ void select_step(const Fp64BandParams& P, int b, const double (&sc)[R],
                                            double (&acc_s)[2 * R - 1], RowSrc& acc_a,
                                            int64_t g0, int lane, double* cslot_s, int* cslot_r) {
    select_rows<R>(b, sc, acc_s, acc_a);
    select_column<R>(P, b, sc, g0, lane, cslot_s, cslot_r);
}

// One chunk = R consecutive columns.  FAST chunks hold only cells of the
// reference's 4-wide (fused) part; each step there evaluates its R cells per
// lane, and the selection runs only when some cell of the warp exceeds its row
// partial or the column's threshold cthr[b] (a warp vote).  Other chunks
// evaluate every cell with its own geometry and always select.  Returns
// whether any step selected (uniform over the warp).
template <int R, bool FAST>
__device__ __forceinline__ bool chunk_fp64(const Fp64BandParams& P, int64_t jc, const char* rring,
                                           const char* rbase, int tbase, double4 (&rwin)[R], double (&qt)[R],
                                           const int* lgeo,
                                           double (&acc_s)[2 * R - 1], RowSrc& acc_a,
                                           int64_t g0, int lane, double* cslot_s, int* cslot_r,
                                           const double* cthr, const char* ccur) {
    bool selected = !FAST;
#pragma unroll
    for (int b = 0; b < R; ++b) {
        const int64_t j = jc + b;
        // record tbase + b + R - 1 (tbase = jc + lane*R): with R = 8 the slot of
        // record tbase + R - 1 is 7 mod 8 and the step offsets are constants
        if (R == 8)
            rwin[(b + R - 1) % R] = ring_rec(rbase + rec_step<7>(b));
        else
            rwin[(b + R - 1) % R] =
                ring_rec(rring + rec_off(rec_slot(tbase + b + R - 1)));
        const double4 cv = ring_rec(ccur + 32 * b);  // column record, staged a chunk ahead
        double sc[R];
        if (FAST) {
            const double tc = cthr[b];
#pragma unroll
            for (int a = 0; a < R; ++a) {
                const double4 rv = rwin[(b + a) % R];
                // 4-wide part of the reference kernel (kernels.cpp:206-225)
                const double ss = __dmul_rn(rv.z, cv.z);
                const double mm = __dmul_rn(cv.w, rv.w);
                sc[a] = __fma_rn(qt[a], ss, -mm);
                qt[a] = __fma_rn(-rv.x, cv.x, __fma_rn(rv.y, cv.y, qt[a]));
            }
            const unsigned hits = step_hits<R>(sc, acc_s, b, tc);
            if (hits) {
                selected = true;
                if (hits & 1u) select_rows<R>(b, sc, acc_s, acc_a);
                if (hits & 2u) select_column<R>(P, b, sc, g0, lane, cslot_s, cslot_r);
            }
        } else {
#pragma unroll
            for (int a = 0; a < R; ++a) {
                const double4 rv = rwin[(b + a) % R];
                double score;
                if (j < lgeo[a * 32]) {
                    const double ss = __dmul_rn(rv.z, cv.z);
                    if (j <= lgeo[(R + a) * 32]) {
                        const double mm = __dmul_rn(cv.w, rv.w);
                        score = __fma_rn(qt[a], ss, -mm);
                        qt[a] = __fma_rn(-rv.x, cv.x, __fma_rn(rv.y, cv.y, qt[a]));
                    } else {
                        // scalar remainder (kernels.cpp:282-289), no fusion
                        score = __dsub_rn(__dmul_rn(qt[a], ss), __dmul_rn(rv.w, cv.w));
                        qt[a] = __dsub_rn(__dadd_rn(qt[a], __dmul_rn(rv.y, cv.y)),
                                          __dmul_rn(rv.x, cv.x));
                    }
                } else {
                    score = -DBL_MAX;
                }
                sc[a] = score;
            }
            select_step<R>(P, b, sc, acc_s, acc_a, g0, lane, cslot_s, cslot_r);
        }
    }
    return selected;
}

template <int R>
__device__ __forceinline__ void band_fp64(const Fp64BandParams& P, int64_t band, int lane,
                                          int shard, double* ring_s, int* ring_c, char* rring,
                                          double* cslot_s, int* cslot_r, double* tring,
                                          double* cthr, char* ccol, int* lgeo) {
    constexpr int RING = 32 * R;
    const int64_t gb = P.g_lo + band * (int64_t)RING;
    const int64_t g0 = gb + (int64_t)lane * R;
    const int64_t jmax = P.Tbase - gb;  // length of the band's longest diagonal
    if (jmax <= 0) return;

    // Per diagonal a of the lane: len = its column count, psw = its last
    // column of the reference's 4-wide part (-1: none), kept in the lane's
    // slots of shared memory (lgeo[a*32], lgeo[(R+a)*32]; columns < 2^31,
    // checked by the host): only the chunks near a diagonal's end read them.
    double qt[R];
    int minpsw = INT32_MAX;
#pragma unroll
    for (int a = 0; a < R; ++a) {
        const int64_t g = g0 + a;
        int len = 0, psw = -1;
        if (g < P.g_hi) {
            const int64_t delta = (g - P.blk_origin) % P.B;
            const int64_t T = P.Tbase - (g - delta);
            qt[a] = P.qt0[g - P.g_lo];
            len = (int)(T - delta);
            psw = (delta < (P.B & ~3ll)) ? (int)(T - 4 * (delta / 4 + 1)) : -1;
        } else {
            qt[a] = 0.0;
        }
        lgeo[a * 32] = len;
        lgeo[(R + a) * 32] = psw;
        minpsw = min(minpsw, psw);
    }

    // ring of row partials, slot = (r - gb) mod RING; column slots of a chunk
    for (int k = lane; k < RING; k += 32) {
        ring_s[k] = -DBL_MAX;
        ring_c[k] = 0;
    }
    if (lane < R) cslot_s[lane] = -DBL_MAX;

    // row records of the band (t = row - gb) and their rows' thresholds staged
    // in the warp's shared-memory rings; before chunk jc they hold t < fill
    const uint4* rsrc = reinterpret_cast<const uint4*>(P.rowrec + gb);
    const double* tsrc = P.thr + gb + P.row_key_off;  // threshold of band row t
    const double* csrc = P.thr + P.col_key_off;       // threshold of column j
    int fill = 34 * R;
    for (int i = lane; i < 2 * fill; i += 32) rec_store(rring, i >> 1, i & 1, __ldg(rsrc + i));
    for (int i = lane; i < fill; i += 32) thr_store(tring, i, ld_thr(tsrc + i));
    if (lane < R) cthr[lane] = ld_thr(csrc + lane);
    // column records of a chunk in shared memory, double-buffered: R records of
    // 32 bytes per buffer, the next chunk's loaded while this one runs
    const uint4* csrc_rec = reinterpret_cast<const uint4*>(P.colrec);
    if (lane < 2 * R) *reinterpret_cast<uint4*>(ccol + 16 * lane) = __ldg(csrc_rec + lane);
    int cbuf = 0;
    __syncwarp();
    // register window of row records: slot (k mod R) holds row g0 + jc + k
    double4 rwin[R];
#pragma unroll
    for (int k = 0; k < R - 1; ++k) rwin[k] = ring_rec(rring + rec_off(rec_slot(lane * R + k)));
    // row partials: slot k holds row g0 + jc + k, starting at the row's
    // threshold with no source (no candidate yet)
    double acc_s[2 * R - 1];
    RowSrc acc_a{0ull};
#pragma unroll
    for (int k = 0; k < 2 * R - 1; ++k) {
        acc_s[k] = tring[thr_off(lane * R + k)];
    }

    bool sel_prev = false;
    for (int64_t jc = 0; jc < jmax; jc += R) {
        // Prefetch what the next chunk appends -- R row records and their
        // rows' thresholds into ring slots this chunk does not read (it reads
        // rows below fill - 1), R column records and column thresholds into
        // the other buffers -- copied straight into shared memory while the
        // chunk runs.  A threshold copied through L1 may be older than the
        // value in L2; any value it has held is a valid lower bound.
        if (lane < 2 * R) {
            const int sr = rec_slot(fill + (lane >> 1));
            const uint4* src = rsrc + 2 * fill + lane;
            cp_async16(rring + rec_off(sr) + 16 * (lane & 1), src);
            if (sr < kRecMirror) cp_async16(rring + rec_off(sr + kRecRing) + 16 * (lane & 1), src);
            cp_async16(ccol + (cbuf ^ 1) * (32 * R) + 16 * lane, csrc_rec + 2 * (jc + R) + lane);
        }
        if (lane < R) {
            const int st = (fill + lane) % kRecRing;
            cp_async8(tring + thr_pos(st), tsrc + fill + lane);
            if (st < kThrMirror) cp_async8(tring + thr_pos(st + kRecRing), tsrc + fill + lane);
            cp_async8(cthr + (cbuf ^ 1) * R + lane, csrc + jc + R + lane);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        const char* ccur = ccol + cbuf * (32 * R);
        const int tbase = (int)jc + lane * R;
        const char* rbase = rring + rec_off(rec_slot(tbase + R - 1));
        const bool fast = __all_sync(kFullMask, jc + R - 1 <= minpsw);
        bool sel;
        if (fast)
            sel = chunk_fp64<R, true>(P, jc, rring, rbase, tbase, rwin, qt, lgeo, acc_s, acc_a,
                                      g0, lane, cslot_s, cslot_r, cthr + cbuf * R, ccur);
        else
            sel = chunk_fp64<R, false>(P, jc, rring, rbase, tbase, rwin, qt, lgeo, acc_s, acc_a,
                                       g0, lane, cslot_s, cslot_r, cthr + cbuf * R, ccur);
        __syncwarp();
        // the chunk's column maxima (one per column, parked by the winning lane)
        if (sel && lane < R) {
            const double cs = cslot_s[lane];
            if (cs > P.floor)
                flush_fp64(P, shard, jc + lane + P.col_key_off, cs,
                           jc + cslot_r[lane] + P.row_nb_off);
            cslot_s[lane] = -DBL_MAX;
        }
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        cbuf ^= 1;
        fill += R;
        // rows jc + g0 + [0, R) are done for this lane: merge its candidates
        // (selected in this chunk or the previous one) into the ring
        if (sel || sel_prev) {
            const int base = (int)(((jc / R) + lane) % 32) * R;
#pragma unroll
            for (int k = 0; k < R; ++k) {
                const int a = acc_a.get(k);
                if (a >= 0 && acc_s[k] > ring_s[base + k]) {
                    ring_s[base + k] = acc_s[k];
                    ring_c[base + k] = (int)(jc + k - a);
                }
            }
        }
        sel_prev = sel;
        __syncwarp();
        // rows jc + gb + [0, R) have now met every lane: flush and free
        if (lane < R) {
            const int e = (int)((jc / R) % 32) * R + lane;
            const double s = ring_s[e];
            if (s > P.floor) flush_fp64(P, shard, jc + gb + lane + P.row_key_off, s,
                                     ring_c[e] + P.col_nb_off);
            ring_s[e] = -DBL_MAX;
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < R - 1; ++k) acc_s[k] = acc_s[k + R];
        acc_a.w >>= 4 * R;  // and the new rows' nibbles are 0
        // new rows jc + R + g0 + k start at their thresholds
        if (R == 8) {
            // rows tbase + 8 + k: slot s0 + k with s0 = (tbase + 8) % kRecRing a
            // multiple of 8 and k < 16 (the mirror keeps them from wrapping)
            const double* tb = tring + thr_pos((tbase + 8) % kRecRing);
#pragma unroll
            for (int k = R - 1; k < 2 * R - 1; ++k) {
                acc_s[k] = tb[k + (k >> 3)];
            }
        } else {
#pragma unroll
            for (int k = R - 1; k < 2 * R - 1; ++k) {
                acc_s[k] = tring[thr_off(tbase + R + k)];
            }
        }
    }

    // drain: carried rows jend + g0 + [0, R-1) into the ring, then every slot
    const int64_t jend = ((jmax + R - 1) / R) * R;
    const int base = (int)(((jend / R) + lane) % 32) * R;
#pragma unroll
    for (int k = 0; k < R - 1; ++k) {
        const int a = acc_a.get(k);
        if (a >= 0 && acc_s[k] > ring_s[base + k]) {
            ring_s[base + k] = acc_s[k];
            ring_c[base + k] = (int)(jend + k - a);
        }
    }
    __syncwarp();
    for (int e = lane; e < RING; e += 32) {
        const double s = ring_s[e];
        if (s > P.floor) {
            const int64_t rel = ((int64_t)e - jend % RING + RING) % RING;
            flush_fp64(P, shard, jend + gb + rel + P.row_key_off, s, ring_c[e] + P.col_nb_off);
        }
    }
    __syncwarp();

    if (P.qt_out) {
#pragma unroll
        for (int a = 0; a < R; ++a)
            if (g0 + a < P.g_hi) P.qt_out[g0 + a - P.g_lo] = qt[a];
    }
}

template <int R>
constexpr int fp64_smem_bytes() {
    return kFp64WarpsPerBlock *
           (kRecRingBytes + 2 * 32 * R + (32 * R + R) * (int)(sizeof(double) + sizeof(int)) +
            (kThrRingDoubles + 2 * R) * (int)sizeof(double) + 2 * R * 32 * (int)sizeof(int));
}

template <int R>
__global__ void __launch_bounds__(32 * kFp64WarpsPerBlock) fp64_band_kernel(const Fp64BandParams P) {
    extern __shared__ __align__(128) char smem_fp64[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    constexpr int kW = kFp64WarpsPerBlock;
    char* p = smem_fp64;
    char* rring = p + w * kRecRingBytes;
    p += kW * kRecRingBytes;
    char* ccol = p + w * (2 * 32 * R);
    p += kW * 2 * 32 * R;
    double* tring = reinterpret_cast<double*>(p) + w * kThrRingDoubles;
    p += kW * kThrRingDoubles * sizeof(double);
    double* ring_s = reinterpret_cast<double*>(p) + w * 32 * R;
    p += kW * 32 * R * sizeof(double);
    double* cslot_s = reinterpret_cast<double*>(p) + w * R;
    p += kW * R * sizeof(double);
    double* cthr = reinterpret_cast<double*>(p) + w * 2 * R;  // two buffers of R
    p += kW * 2 * R * sizeof(double);
    int* ring_c = reinterpret_cast<int*>(p) + w * 32 * R;
    p += kW * 32 * R * sizeof(int);
    int* cslot_r = reinterpret_cast<int*>(p) + w * R;
    p += kW * R * sizeof(int);
    int* lgeo = reinterpret_cast<int*>(p) + w * 2 * R * 32 + lane;
    // One resident wave of W warps.  Band b (longest first: band lengths fall
    // with b) goes to warp b mod W in even rounds and W-1 - (b mod W) in odd
    // rounds, so every warp's bands add up to nearly the same length -- the
    // reference's (k, nbands-1-k) pairing carried over any number of rounds.
    const int64_t W = (int64_t)gridDim.x * kFp64WarpsPerBlock;
    const int64_t wid = (int64_t)blockIdx.x * kFp64WarpsPerBlock + w;
    const int shard = (int)(wid % P.shards);
    for (int64_t r = 0;; ++r) {
        const int64_t band = r * W + ((r & 1) ? W - 1 - wid : wid);
        if (band >= P.nbands) break;
        band_fp64<R>(P, band, lane, shard, ring_s, ring_c, rring, cslot_s, cslot_r, tring, cthr,
                     ccol, lgeo);
    }
}

}  // namespace

template <int R>
void launch_fp64_band(const Fp64BandParams& P, cudaStream_t s) {
    constexpr int smem = fp64_smem_bytes<R>();
    // per-device attribute and occupancy, idempotent: see launch_fp32_join
    static std::atomic<unsigned long long> configured{0};
    static std::atomic<int> resident[64];
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load(std::memory_order_acquire) & bit)) {
        cudaFuncSetAttribute(fp64_band_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fp64_band_kernel<R>,
                                                          32 * kFp64WarpsPerBlock, smem) != cudaSuccess ||
            per_sm < 1) {
            cudaGetLastError();
            per_sm = 1;
        }
        resident[dev & 63].store(per_sm, std::memory_order_relaxed);
        configured.fetch_or(bit, std::memory_order_release);
    }
    // one resident wave, fewer CTAs when there are fewer bands than warps
    const int64_t wave = (int64_t)sm_count() * resident[dev & 63].load(std::memory_order_relaxed);
    const int64_t want = (P.nbands + kFp64WarpsPerBlock - 1) / kFp64WarpsPerBlock;
    const int64_t blocks = std::min<int64_t>(want, wave);
    if (blocks > 0) fp64_band_kernel<R><<<(unsigned)blocks, 32 * kFp64WarpsPerBlock, smem, s>>>(P);
}

template void launch_fp64_band<1>(const Fp64BandParams&, cudaStream_t);
template void launch_fp64_band<2>(const Fp64BandParams&, cudaStream_t);
template void launch_fp64_band<4>(const Fp64BandParams&, cudaStream_t);
template void launch_fp64_band<8>(const Fp64BandParams&, cudaStream_t);

}  // namespace mpgpu
