// FP32 re-anchored tile join.
//
// The distance matrix is cut into tiles of 32*R adjacent diagonals (one
// band) by K columns.  A warp owns one tile: lane l owns diagonals
// g0 + a (a < R, g0 = band start + l*R), all lanes walk the tile's columns
// together.
//
//  anchor     at the tile's first column j0 each lane computes the exact
//             covariance of its R window pairs in FP64:
//               cov = sum_k A[j0+k]*A[j0+g+k] - m*mean[j0]*mean[j0+g]
//             (the re-anchor; one per K recurrence steps);
//  recurrence the centred update of SCAMP (Zimmerman et al., SoCC 2019),
//               cov(j+1, r+1) = cov(j, r) + df[j]*dg[r] + df[r]*dg[j],
//             in FP32 on the Blackwell f32x2 datapath: diagonals a and a+R/2
//             share one 64-bit register pair, so every fma/mul instruction
//             advances two cells;
//  distance   u = 1 - cov*nn[j]*nn[r] (= d^2 / 2m) as a single fused op;
//  min/argmin the low 8 bits of u's bit pattern are replaced by the cell's
//             position in the band (lane<<3 | a), so one float min tracks
//             value and origin at once (2^-15 relative resolution, far
//             inside the 1e-4 target).  Rows accumulate in registers for R
//             steps (columns go in pairs, so one 3-input min takes a cell
//             of each column) and then in a per-warp shared-memory ring; a column's
//             warp minimum is one REDUX instruction.  Finished rows/columns
//             are merged into the profile with a 64-bit atomicMin on
//             (ordered u, neighbour).
//  group keys (the guarded form) a lane takes plain float minima over its
//             own cells, and only the lane's results carry the lane number
//             in their low 8 bits (one tag per row or column, not per cell);
//             a key then names the winning lane's R adjacent candidate
//             neighbours, among which the finalisation picks with FP64 dot
//             products (fp32_pick_neighbour) -- which also removes FP32
//             ranking noise between adjacent diagonals.
//
// Reference semantics kept: strict improvement over the initial score -1
// (u < 1 + 1/m), NaN never wins (a zero-variance window has nn = NaN).
#include <algorithm>
#include <atomic>

#include "mp_common.cuh"
#include "mp_kernels.h"

namespace mpgpu {

namespace {

// A row record in memory (global and the shared-memory ring): 32 bytes.
struct RowRec {
    float4 dfdg;  // (df[j], df[j+H], dg[j], dg[j+H])
    float4 nn1;   // (nn[j], nn[j+H], 1, 1)
};
// The part of a row record a lane keeps in registers (the constant pair stays
// behind: one shared (1, 1) operand serves every fused distance).
struct RowWin {
    float4 dfdg;
    float2 nn;
};
__device__ __forceinline__ float2 lo2(const float4& v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(const float4& v) { return make_float2(v.z, v.w); }
static_assert(sizeof(RowRec) == 32, "row record is 32 bytes");

constexpr unsigned kTagMask = 0xffu;
constexpr float kInf = __builtin_huge_valf();

// Row-partial ring: 34 chunks of 8 rows, 12 floats apart (48 bytes), so that
// the 8 lanes of a quarter-warp merging their chunks with 16-byte accesses
// hit 8 distinct groups of 4 banks (a 32-byte stride would pair them up).
constexpr int kRowChunks = 34;
constexpr int kRowStride = 12;

// Terms of the FP64 anchor staged per pass: the column's chunk plus the warp's
// 32*8 + chunk rows (skewed by 1/8) must fit the record ring.
constexpr int kAnchorChunk = 512;
static_assert(8 * (kAnchorChunk + (32 * 8 + kAnchorChunk) * 9 / 8) <= kRecRingBytes,
              "anchor staging fits the record ring");

// 16-byte copy global -> shared that completes asynchronously (cp.async.cg:
// cached in L2 only); both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(char* dst_smem, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ float tag_key(float u, unsigned tag) {
    return __uint_as_float((__float_as_uint(u) & ~kTagMask) | tag);
}
__device__ __forceinline__ float untag_value(unsigned bits) {
    return __uint_as_float((bits & ~kTagMask) | 0x80u);
}
// u with the lane number in its low 8 bits (group keys: a lane's minima only).
__device__ __forceinline__ float tag_lane(float u, unsigned lane) {
    return __uint_as_float((__float_as_uint(u) & ~kTagMask) | lane);
}

template <bool GROUP>
__device__ __forceinline__ float lane_min(float v, int lane) {
    return GROUP ? tag_lane(v, (unsigned)lane) : v;
}

// Group keys: merges (u, candidates [base, base + count)) unless u is not
// below the initial score's ulim.
__device__ __forceinline__ void merge_group(unsigned long long* key, float u, int64_t base,
                                            int count, unsigned ulim_ord) {
    const unsigned hi = (ord_f32(u) & ~kTagMask) | 0x80u | (unsigned)(count - 1);
    if (hi < ulim_ord)
        atomicMin(key, ((unsigned long long)hi << 32) | kFp32GroupBit | (unsigned long long)base);
}
// Row r's minimum over the band, tagged with its lane L: the cells of lane L
// in row r are (j = r - g, g = gL + a) for a < R with g < g_hi and j >= 0,
// gL = gb + L*R, i.e. the columns [r - gL - amax, r - gL].  WHOLE: the tile
// guarantees amax = R - 1 for every lane (see tile_fp32).
template <int R, bool WHOLE>
__device__ __forceinline__ void flush_row_group(const Fp32TileParams& P, float v, int64_t r,
                                                int64_t gb, unsigned ulim_ord) {
    const unsigned bits = __float_as_uint(v);
    const float u = untag_value(bits);
    if (!(u < kInf)) return;  // no cell (kInf or a NaN pattern)
    const int64_t gL = gb + (int64_t)(bits & kTagMask) * R;
    const int64_t amax = WHOLE ? (int64_t)R - 1 : min(min((int64_t)R - 1, P.g_hi - 1 - gL), r - gL);
    merge_group(P.key + r, u, r - gL - amax, (int)amax + 1, ulim_ord);
}
// Column j's minimum over the band, tagged with its lane L: the candidates
// are rows j + gL + a, a < R, on diagonals < g_hi and rows < PL.  WHOLE: the
// tile guarantees all R of them for every lane.
template <int R, bool WHOLE>
__device__ __forceinline__ void flush_col_group(const Fp32TileParams& P, unsigned bits, int64_t j,
                                                int64_t gb, unsigned ulim_ord) {
    const float u = untag_value(bits);
    if (!(u < kInf)) return;
    const int64_t gL = gb + (int64_t)(bits & kTagMask) * R;
    const int64_t cnt = WHOLE ? (int64_t)R : min(min((int64_t)R, P.g_hi - gL), P.PL - j - gL);
    merge_group(P.key + j, u, j + gL, (int)cnt, ulim_ord);
}

template <int R>
__device__ __forceinline__ void flush_row(const Fp32TileParams& P, float v, int64_t r,
                                          int64_t gb, float ulim) {
    const unsigned bits = __float_as_uint(v);
    const float u = untag_value(bits);
    if (u < ulim) {
        const unsigned t = bits & kTagMask;
        const int64_t dw = (int64_t)(t >> 3) * R + (t & 7u);
        const int64_t j = r - (gb + dw);
        atomicMin(P.key + r, ((unsigned long long)ord_f32(u) << 32) | (unsigned long long)j);
    }
}

// One chunk = R consecutive columns.  Per column: R cells per lane, the
// lane's column minimum, then one warp-wide REDUX; lane OFF + b keeps the
// result of column b so the column flushes happen once per chunk pair, with
// no divergent branch between steps (consecutive steps can overlap).  Row
// partials live in a 2R-entry circular register array; OFF (0 or R) is the
// chunk's rotation, so no register ever moves between chunks.
// Slow chunks (near the end of a band) mask cells past the diagonal's end:
// cell (column jr + b, diagonal g0 + d) exists iff d < ghi_rel and
// jr + b < min(lim0 - d, ncols).
template <int R, bool FAST, int OFF, bool GROUP>
__device__ __forceinline__ void chunk_fp32(const char* rbase, const char* cbuf,
                                           RowWin (&win)[R / 2], float2 (&nc2)[R / 2],
                                           float (&acc)[2 * R], const unsigned (&tag)[R],
                                           int lim0, int ncols, int ghi_rel, int jr, int lane,
                                           int& colkey) {
    constexpr int H = R / 2;
    static_assert(R % 2 == 0, "columns are processed in pairs");
    const float2 one2 = make_float2(1.f, 1.f);
    // Columns go in pairs (b, b + 1): row slot s = b + d takes cell d of
    // column b and cell d - 1 of column b + 1, so one 3-input min per slot
    // serves both columns (9 row-min instructions per 2R cells, not 2R).
#pragma unroll
    for (int b = 0; b < R; b += 2) {
        float kb[R];  // column b's tagged cells, by diagonal
        {
            {
                // record tbase + b + H - 1; tbase % 8 == 0, so its slot % 8 == H - 1
                const char* p = rbase + rec_step<H - 1>(b);
                win[(b + H - 1) % H].dfdg = *reinterpret_cast<const float4*>(p);
                win[(b + H - 1) % H].nn = *reinterpret_cast<const float2*>(p + 16);
            }
            const float4 cv = *reinterpret_cast<const float4*>(cbuf + 32 * b);
            const float2 cnn = *reinterpret_cast<const float2*>(cbuf + 32 * b + 16);
            float cmin;
#pragma unroll
            for (int a = 0; a < H; ++a) {
                const RowWin& rv = win[(b + a) % H];
                const float2 nn2 = __fmul2_rn(cnn, rv.nn);
                const float2 u2 = __ffma2_rn(nc2[a], nn2, one2);
                nc2[a] = __ffma2_rn(lo2(cv), hi2(rv.dfdg), nc2[a]);
                nc2[a] = __ffma2_rn(lo2(rv.dfdg), hi2(cv), nc2[a]);
                kb[a] = GROUP ? u2.x : tag_key(u2.x, tag[a]);
                kb[a + H] = GROUP ? u2.y : tag_key(u2.y, tag[a + H]);
                if (!FAST) {
                    const int l0 = a < ghi_rel ? min(lim0 - a, ncols) : 0;
                    const int l1 = a + H < ghi_rel ? min(lim0 - a - H, ncols) : 0;
                    if (jr + b >= l0) kb[a] = kInf;
                    if (jr + b >= l1) kb[a + H] = kInf;
                }
                cmin = a == 0 ? fminf(kb[a], kb[a + H]) : fmin3(cmin, kb[a], kb[a + H]);
            }
            acc[(b + OFF) % (2 * R)] = fminf(acc[(b + OFF) % (2 * R)], kb[0]);
            const int kmin =
                __reduce_min_sync(kFullMask, __float_as_int(GROUP ? tag_lane(cmin, lane) : cmin));
            colkey = (lane == b + OFF) ? kmin : colkey;
        }
        {
            const int c = b + 1;
            {
                const char* p = rbase + rec_step<H - 1>(c);
                win[(c + H - 1) % H].dfdg = *reinterpret_cast<const float4*>(p);
                win[(c + H - 1) % H].nn = *reinterpret_cast<const float2*>(p + 16);
            }
            const float4 cv = *reinterpret_cast<const float4*>(cbuf + 32 * c);
            const float2 cnn = *reinterpret_cast<const float2*>(cbuf + 32 * c + 16);
            float cmin;
#pragma unroll
            for (int a = 0; a < H; ++a) {
                const RowWin& rv = win[(c + a) % H];
                const float2 nn2 = __fmul2_rn(cnn, rv.nn);
                const float2 u2 = __ffma2_rn(nc2[a], nn2, one2);
                nc2[a] = __ffma2_rn(lo2(cv), hi2(rv.dfdg), nc2[a]);
                nc2[a] = __ffma2_rn(lo2(rv.dfdg), hi2(cv), nc2[a]);
                float k0 = GROUP ? u2.x : tag_key(u2.x, tag[a]);
                float k1 = GROUP ? u2.y : tag_key(u2.y, tag[a + H]);
                if (!FAST) {
                    const int l0 = a < ghi_rel ? min(lim0 - a, ncols) : 0;
                    const int l1 = a + H < ghi_rel ? min(lim0 - a - H, ncols) : 0;
                    if (jr + c >= l0) k0 = kInf;
                    if (jr + c >= l1) k1 = kInf;
                }
                // slot c + a: cell a of column c and cell a + 1 of column b
                acc[(c + a + OFF) % (2 * R)] = fmin3(acc[(c + a + OFF) % (2 * R)], k0, kb[a + 1]);
                // slot c + a + H: cell a + H of column c and cell a + H + 1 of column
                // b.  Slots b + R - 1 and b + R begin new rows here (these are their
                // first cells), so they are assigned and no slot needs a reset.
                if (a == H - 1)
                    acc[(c + a + H + OFF) % (2 * R)] = k1;
                else if (a == H - 2)
                    acc[(c + a + H + OFF) % (2 * R)] = fminf(k1, kb[a + H + 1]);
                else
                    acc[(c + a + H + OFF) % (2 * R)] =
                        fmin3(acc[(c + a + H + OFF) % (2 * R)], k1, kb[a + H + 1]);
                cmin = a == 0 ? fminf(k0, k1) : fmin3(cmin, k0, k1);
            }
            const int kmin =
                __reduce_min_sync(kFullMask, __float_as_int(GROUP ? tag_lane(cmin, lane) : cmin));
            colkey = (lane == c + OFF) ? kmin : colkey;
        }
    }
}

template <int R, bool GROUP>
__device__ void tile_fp32(const Fp32TileParams& P, int64_t band, int64_t seg, int lane, float* ring,
                          char* rring, char* cring) {
    constexpr int H = R / 2;
    constexpr int RING = 32 * R;
    const int64_t gb = P.g_lo + band * (int64_t)RING;
    const int64_t g0 = gb + (int64_t)lane * R;
    const int64_t jmax = P.PL - gb;
    const int64_t j0 = seg * P.K;
    const int64_t j1 = min(j0 + P.K, jmax);
    if (j0 >= j1) return;
    // guarded form: tiles touching a hazard window are evaluated in FP64
    if (P.hazard && fp32_tile_hazardous(P, gb, j0, j1, 32 * R)) return;
    const float ulim = (float)(1.0 + 1.0 / (double)P.m);
    const unsigned ulim_ord = ord_f32(ulim);
    // group keys: every lane's candidate groups hold all R candidates (its
    // diagonals lie below g_hi, rows below PL, and columns, j0 >= R - 1, at or
    // above 0)
    const bool whole = j0 >= R - 1 && gb + 32 * R <= P.g_hi && j1 + gb + 32 * R <= P.PL;

    // cell (column j, diagonal g0 + d) is evaluated iff d < ghi_rel and
    // j - j0 < min(lim0 - d, ncols); every cell of a chunk ending at or
    // before minlim exists
    const int ncols = (int)(j1 - j0);
    const int lim0 = (int)min(P.PL - g0 - j0, (int64_t)ncols + R);
    const int ghi_rel = (int)max(min(P.g_hi - g0, (int64_t)R), (int64_t)0);
    const int minlim = ghi_rel < R ? 0 : min(lim0 - (R - 1), ncols);
    // tag of cell d: lane << 3 | d
    unsigned tag[R];
#pragma unroll
    for (int a = 0; a < R; ++a) tag[a] = ((unsigned)lane << 3) | (unsigned)a;

    // ---- FP64 re-anchor: cov(j0, j0+g) for the lane's R diagonals ----------
    // The series terms are staged in the (not yet used) record ring with
    // coalesced loads, kAnchorChunk terms at a time: the column's A[j0 + k]
    // and the warp's rows A[j0 + gb + i], i < 32R + chunk, skewed by one double
    // per 8 so that lanes reading rows 8 apart hit distinct banks.  Each lane
    // then sums its R products in k order from shared memory.
    double mu0 = (double)P.m * __ldg(P.mean + j0);
    double mr[R];
#pragma unroll
    for (int a = 0; a < R; ++a) mr[a] = __ldg(P.mean + j0 + g0 + a);
    double q[R];
#pragma unroll
    for (int a = 0; a < R; ++a) q[a] = 0.0;
    {
        static_assert(R % 8 == 0, "anchor row skew assumes lanes start on multiples of 8 rows");
        double* scol = reinterpret_cast<double*>(rring);
        double* srow = scol + kAnchorChunk;
        const double* Ac = P.A + j0;
        const double* Ar = P.A + j0 + gb;
        // lane's rows i = lane*R + t sit at srow[lane*(R + R/8) + t + t/8]
        const double* wl = srow + lane * (R + R / 8);
        for (int64_t kb0 = 0; kb0 < P.m; kb0 += kAnchorChunk) {
            const int kc = (int)min((int64_t)kAnchorChunk, P.m - kb0);
            __syncwarp();
#pragma unroll 4
            for (int i = lane; i < kc; i += 32) scol[i] = __ldg(Ac + kb0 + i);
#pragma unroll 4
            for (int i = lane; i < 32 * R + kc; i += 32) srow[i + (i >> 3)] = __ldg(Ar + kb0 + i);
            __syncwarp();
            double w[R];
#pragma unroll
            for (int a = 0; a < R - 1; ++a) w[a] = wl[a];
            int k = 0;
            for (; k + R <= kc; k += R) {
                const double* wk = wl + (k / 8) * 9;  // row lane*R + k, k % 8 == 0
#pragma unroll
                for (int kk = 0; kk < R; ++kk) {
                    const int t = kk + R - 1;
                    w[(kk + R - 1) % R] = wk[t + (t >> 3)];
                    const double x = scol[k + kk];
#pragma unroll
                    for (int a = 0; a < R; ++a) q[a] = __fma_rn(x, w[(kk + a) % R], q[a]);
                }
            }
            for (; k < kc; ++k) {
                const double x = scol[k];
#pragma unroll
                for (int a = 0; a < R; ++a) {
                    const int t = k + a;
                    q[a] = __fma_rn(x, wl[t + (t >> 3)], q[a]);
                }
            }
        }
        __syncwarp();
    }
    float2 nc2[H];
    {
        float nc[R];
#pragma unroll
        for (int a = 0; a < R; ++a) nc[a] = (float)__fma_rn(mu0, mr[a], -q[a]);
#pragma unroll
        for (int a = 0; a < H; ++a) nc2[a] = make_float2(nc[a], nc[a + H]);
    }

    // ---- ring of row partials for this tile -----------------------------------
    for (int k = lane; k < kRowChunks * kRowStride; k += 32) ring[k] = kInf;
    __syncwarp();

    // row partials: row o of chunk c (o in [0, 2R-1)) lives in acc[(o + R*(c%2)) % 2R]
    float acc[2 * R];
#pragma unroll
    for (int k = 0; k < 2 * R; ++k) acc[k] = kInf;

    // row records of the band, tile-relative index t = row - (j0 + gb), staged
    // in the warp's shared-memory ring; before chunk pair i it holds t < fill
    const uint4* rsrc = reinterpret_cast<const uint4*>(
        reinterpret_cast<const RowRec*>(P.rowrec) + (j0 + gb));
    int fill = 33 * R + H;
    for (int i = lane; i < 2 * fill; i += 32) rec_store(rring, i >> 1, i & 1, __ldg(rsrc + i));
    // column records of a chunk pair (2R records), double-buffered
    const uint4* csrc = reinterpret_cast<const uint4*>(
        reinterpret_cast<const RowRec*>(P.colrec) + j0);
    *reinterpret_cast<uint4*>(cring + 16 * lane) = __ldg(csrc + lane);
    __syncwarp();
    RowWin win[H];
#pragma unroll
    for (int k = 0; k < H - 1; ++k) {
        const char* p = rring + rec_off(rec_slot(lane * R + k));
        win[k].dfdg = *reinterpret_cast<const float4*>(p);
        win[k].nn = *reinterpret_cast<const float2*>(p + 16);
    }

    // Row partials leave the registers through a ring of kRowChunks chunks of
    // R rows in shared memory: row t of the tile sits at
    // ((t / R) % kRowChunks) * kRowStride + t % R.  With 34 chunks the rows
    // finished by lane 0 in a chunk pair stay put until they are flushed at the
    // end of the pair.
    constexpr int RK_CHUNKS = kRowChunks;
    static_assert(R == 8, "row ring stride is laid out for 8 rows per chunk");
    int cb = 0;                              // column buffer of the current pair
    int rslot = rec_slot(lane * R + H - 1);  // record slot of jr + lane*R + H - 1
    int kslot = lane;                        // (jr / R + lane) % RK_CHUNKS
    int jr = 0;
    for (; jr < ncols; jr += 2 * R) {
        // prefetch what the next pair appends, 2R row records (ring slots this
        // pair does not read: the ring holds 33R + H + 2R < kRecRing records
        // from the pair's first) and 2R column records (the other buffer),
        // copied straight into shared memory while the pair runs
        {
            const int s = rec_slot(fill + (lane >> 1));
            const uint4* src = rsrc + 2 * fill + lane;
            cp_async16(rring + rec_off(s) + 16 * (lane & 1), src);
            if (s < kRecMirror) cp_async16(rring + rec_off(s + kRecRing) + 16 * (lane & 1), src);
            cp_async16(cring + (cb ^ 1) * 64 * R + 16 * lane, csrc + 2 * (jr + 2 * R) + lane);
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        }
        int colkey = 0x7fffffff;
        const char* cbuf = cring + cb * 64 * R;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int jh = jr + half * R;
            const char* rbase = rring + rec_off(rslot);
            rslot += R;
            if (rslot >= kRecRing) rslot -= kRecRing;
            const bool fast = __all_sync(kFullMask, jh + R <= minlim);
            if (half == 0) {
                if (fast)
                    chunk_fp32<R, true, 0, GROUP>(rbase, cbuf, win, nc2, acc, tag, lim0, ncols, ghi_rel, jh, lane, colkey);
                else
                    chunk_fp32<R, false, 0, GROUP>(rbase, cbuf, win, nc2, acc, tag, lim0, ncols, ghi_rel, jh, lane, colkey);
            } else {
                if (fast)
                    chunk_fp32<R, true, R, GROUP>(rbase, cbuf + 32 * R, win, nc2, acc, tag, lim0,
                                           ncols, ghi_rel, jh, lane, colkey);
                else
                    chunk_fp32<R, false, R, GROUP>(rbase, cbuf + 32 * R, win, nc2, acc, tag,
                                            lim0, ncols, ghi_rel, jh, lane, colkey);
            }
            // this chunk's lower half (rows jh + g0 + [0, R)) is final for the lane
            const int ks = (kslot + half) >= RK_CHUNKS ? kslot + half - RK_CHUNKS : kslot + half;
            float4* rv4 = reinterpret_cast<float4*>(ring + ks * kRowStride);
#pragma unroll
            for (int v = 0; v < R / 4; ++v) {
                float4 t = rv4[v];
                t.x = fminf(t.x, lane_min<GROUP>(acc[(4 * v + 0 + half * R) % (2 * R)], lane));
                t.y = fminf(t.y, lane_min<GROUP>(acc[(4 * v + 1 + half * R) % (2 * R)], lane));
                t.z = fminf(t.z, lane_min<GROUP>(acc[(4 * v + 2 + half * R) % (2 * R)], lane));
                t.w = fminf(t.w, lane_min<GROUP>(acc[(4 * v + 3 + half * R) % (2 * R)], lane));
                rv4[v] = t;
            }
            // lane l's next merge reads the chunk lane l + 1 has just written
            __syncwarp();
        }
        kslot += 2;
        if (kslot >= RK_CHUNKS) kslot -= RK_CHUNKS;
        __syncwarp();
        // columns jr + [0, 2R): one per lane
        if (lane < 2 * R) {
            if constexpr (GROUP) {
                // rows jr + [0, 2R) of the tile have met every lane: flush, free
                const int c = jr / R + (lane >> 3);
                const int e = (c % RK_CHUNKS) * kRowStride + (lane & (R - 1));
                const float v = ring[e];
                ring[e] = kInf;
                const int64_t j = j0 + jr + lane, r = j0 + gb + jr + lane;
                if (whole) {
                    flush_col_group<R, true>(P, (unsigned)colkey, j, gb, ulim_ord);
                    flush_row_group<R, true>(P, v, r, gb, ulim_ord);
                } else {
                    flush_col_group<R, false>(P, (unsigned)colkey, j, gb, ulim_ord);
                    flush_row_group<R, false>(P, v, r, gb, ulim_ord);
                }
            } else {
                const unsigned bits = (unsigned)colkey;
                const float u = untag_value(bits);
                if (u < ulim) {
                    const unsigned t = bits & kTagMask;
                    const int64_t j = j0 + jr + lane;
                    const int64_t q = j + gb + (int64_t)(t >> 3) * R + (t & 7u);
                    atomicMin(P.key + j, ((unsigned long long)ord_f32(u) << 32) | (unsigned long long)q);
                }
                // rows jr + [0, 2R) of the tile have met every lane: flush, free
                const int c = jr / R + (lane >> 3);
                const int e = (c % RK_CHUNKS) * kRowStride + (lane & (R - 1));
                const float v = ring[e];
                ring[e] = kInf;
                flush_row<R>(P, v, j0 + gb + jr + lane, gb, ulim);
            }
        }
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        cb ^= 1;
        fill += 2 * R;
        __syncwarp();
    }

    // drain: the carried upper half (rows jr + lane*R + [0, R-1)), then every slot
    {
        float* base = ring + kslot * kRowStride;
#pragma unroll
        for (int k = 0; k < R - 1; ++k) base[k] = fminf(base[k], lane_min<GROUP>(acc[k], lane));
    }
    __syncwarp();
    const int cend = jr / R;
    for (int e = lane; e < RK_CHUNKS * R; e += 32) {
        const int cs = e / R;
        const int rel = (cs - cend % RK_CHUNKS + RK_CHUNKS) % RK_CHUNKS;
        const int64_t r = j0 + gb + (int64_t)(cend + rel) * R + (e % R);
        if constexpr (GROUP)
            flush_row_group<R, false>(P, ring[cs * kRowStride + e % R], r, gb, ulim_ord);
        else
            flush_row<R>(P, ring[cs * kRowStride + e % R], r, gb, ulim);
    }
    __syncwarp();
}

constexpr int kFp32WarpsPerBlock = 4;

constexpr int kRowKeySlots = kRowChunks * kRowStride;
template <int R>
constexpr int fp32_smem_bytes() {
    return kFp32WarpsPerBlock * (kRecRingBytes + kRowKeySlots * (int)sizeof(float) + 4 * 32 * R);
}

#ifndef MPGPU_FP32_MIN_BLOCKS
#define MPGPU_FP32_MIN_BLOCKS 3  // 3 x 4 warps per SM (measured best of 2, 3, 4)
#endif

// CTAs per SM: group keys need fewer registers (no per-cell tags), and at 4
// CTAs (128 registers) that instantiation ran faster than at 3 (c2 guarded
// join 175 ms against 178); the tagged one spills more there and ran slower.
template <bool GROUP>
constexpr int fp32_blocks_per_sm() {
    return GROUP ? 4 : MPGPU_FP32_MIN_BLOCKS;
}

template <int R, bool GROUP>
__global__ void __launch_bounds__(32 * kFp32WarpsPerBlock, fp32_blocks_per_sm<GROUP>())
    fp32_join_kernel(const Fp32TileParams* __restrict__ series, int nseries, int64_t total,
                     unsigned long long* __restrict__ counter) {
    extern __shared__ __align__(128) char smem_fp32[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    char* rring = smem_fp32 + w * kRecRingBytes;
    float* ring = reinterpret_cast<float*>(smem_fp32 + kFp32WarpsPerBlock * kRecRingBytes) +
                  w * kRowKeySlots;
    char* cring = smem_fp32 + kFp32WarpsPerBlock * (kRecRingBytes + kRowKeySlots * (int)sizeof(float)) +
                  w * 4 * 32 * R;
    // Persistent warps: each takes the next tile number from one global
    // counter until the tile space is exhausted (no waiting on anything).
    for (;;) {
        unsigned long long t0 = 0;
        if (lane == 0) t0 = atomicAdd(counter, 1ull);
        const int64_t tt = (int64_t)__shfl_sync(kFullMask, t0, 0);
        if (tt >= total) break;
        // the series owning tile tt: last descriptor with tile_begin <= tt
        int lo = 0, hi = nseries - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (series[mid].tile_begin <= tt) lo = mid;
            else hi = mid - 1;
        }
        const Fp32TileParams P = series[lo];
        // local tile -> band and column segment (band pairs of nearly equal
        // tile counts); consecutive tiles are consecutive column segments of
        // one band, so tiles running together touch disjoint columns and rows
        int64_t band, seg;
        if (fp32_tile_of(P, tt - P.tile_begin + P.tile_skip, 32 * R, band, seg))
            tile_fp32<R, GROUP>(P, band, seg, lane, ring, rring, cring);
    }
}

}  // namespace

void fp32_tile_plan(int64_t PL, int64_t g_lo, int64_t g_hi, int64_t K, int R, int64_t& nbands,
                    int64_t& seg_per_pair, int64_t& ntiles) {
    const int64_t span = 32 * R;
    const int64_t ndiag = g_hi > g_lo ? g_hi - g_lo : 0;
    nbands = (ndiag + span - 1) / span;
    const int64_t npairs = (nbands + 1) / 2;
    int64_t spp = 0;
    for (int64_t p = 0; p < npairs; ++p) {
        int64_t t = (PL - (g_lo + p * span) + K - 1) / K;
        const int64_t p2 = nbands - 1 - p;
        if (p2 > p) t += (PL - (g_lo + p2 * span) + K - 1) / K;
        spp = std::max(spp, t);
    }
    seg_per_pair = std::max<int64_t>(spp, 1);
    ntiles = npairs * seg_per_pair;
}

template <int R>
void configure_fp32_join() {
    cudaFuncSetAttribute(fp32_join_kernel<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         fp32_smem_bytes<R>());
    cudaFuncSetAttribute(fp32_join_kernel<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         fp32_smem_bytes<R>());
}

template <int R>
void launch_fp32_join(const Fp32TileParams* series_dev, int nseries, int64_t total,
                      unsigned long long* counter, cudaStream_t s, bool group) {
    // the shared-memory limit is a per-device attribute; setting it is
    // idempotent, so concurrent first launches (server threads) are harmless
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(configured.load(std::memory_order_acquire) & bit)) {
        configure_fp32_join<R>();
        configured.fetch_or(bit, std::memory_order_release);
    }
    const int64_t want = (total + kFp32WarpsPerBlock - 1) / kFp32WarpsPerBlock;
    const int64_t blocks = std::min<int64_t>(
        want, (int64_t)sm_count() * (group ? fp32_blocks_per_sm<true>() : fp32_blocks_per_sm<false>()));
    if (blocks > 0 && group)
        fp32_join_kernel<R, true><<<(unsigned)blocks, 32 * kFp32WarpsPerBlock, fp32_smem_bytes<R>(), s>>>(
            series_dev, nseries, total, counter);
    else if (blocks > 0)
        fp32_join_kernel<R, false><<<(unsigned)blocks, 32 * kFp32WarpsPerBlock, fp32_smem_bytes<R>(),
                                     s>>>(series_dev, nseries, total, counter);
}

template void launch_fp32_join<8>(const Fp32TileParams*, int, int64_t, unsigned long long*,
                                  cudaStream_t, bool);
template void configure_fp32_join<8>();

}  // namespace mpgpu
