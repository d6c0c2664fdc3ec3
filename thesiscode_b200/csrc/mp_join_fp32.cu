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
//             steps and then in a per-warp shared-memory ring; a column's
//             warp minimum is one REDUX instruction.  Finished rows/columns
//             are merged into the profile with a 64-bit atomicMin on
//             (ordered u, neighbour).
//
// Reference semantics kept: strict improvement over the initial score -1
// (u < 1 + 1/m), NaN never wins (a zero-variance window has nn = NaN).
#include "mp_common.cuh"
#include "mp_kernels.h"

namespace mpgpu {

namespace {

struct RowRec {
    ulonglong2 dfdg;         // (df[j], df[j+H]), (dg[j], dg[j+H])
    unsigned long long nn;   // (nn[j], nn[j+H])
    unsigned long long pad;
};
static_assert(sizeof(RowRec) == 32, "row record is 32 bytes");

constexpr unsigned kTagMask = 0xffu;
constexpr float kInf = __builtin_huge_valf();

__device__ __forceinline__ float tag_key(float u, unsigned tag) {
    return __uint_as_float((__float_as_uint(u) & ~kTagMask) | tag);
}
__device__ __forceinline__ float untag_value(unsigned bits) {
    return __uint_as_float((bits & ~kTagMask) | 0x80u);
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
// lane's column minimum, then one warp-wide REDUX; lane b keeps the result of
// column b so the chunk's column flushes happen once, after the chunk, with no
// divergent branch between steps (consecutive steps can overlap).
template <int R, bool FAST>
__device__ __forceinline__ void chunk_fp32(const char* rbase, const char* cbuf,
                                           RowRec (&win)[R / 2], unsigned long long (&nc2)[R / 2],
                                           float (&acc)[2 * R - 1], const unsigned (&tag)[R],
                                           const int (&limr)[R], int jr, int lane, int& colkey) {
    constexpr int H = R / 2;
    const unsigned long long one2 = f2_pack(1.0f, 1.0f);
#pragma unroll
    for (int b = 0; b < R; ++b) {
        {
            // record tbase + b + H - 1; tbase % 8 == 0, so its slot % 8 == H - 1
            const char* p = rbase + rec_step<H - 1>(b);
            win[(b + H - 1) % H].dfdg = *reinterpret_cast<const ulonglong2*>(p);
            win[(b + H - 1) % H].nn = *reinterpret_cast<const unsigned long long*>(p + 16);
        }
        const ulonglong2 cdfdg = *reinterpret_cast<const ulonglong2*>(cbuf + 32 * b);
        const unsigned long long cnn = *reinterpret_cast<const unsigned long long*>(cbuf + 32 * b + 16);
        float cmin = kInf;
#pragma unroll
        for (int a = 0; a < H; ++a) {
            const RowRec& rv = win[(b + a) % H];
            const unsigned long long nn2 = f2_mul(cnn, rv.nn);
            const unsigned long long u2 = f2_fma(nc2[a], nn2, one2);
            nc2[a] = f2_fma(cdfdg.x, rv.dfdg.y, nc2[a]);
            nc2[a] = f2_fma(rv.dfdg.x, cdfdg.y, nc2[a]);
            float u0, u1;
            f2_unpack(u2, u0, u1);
            float k0 = tag_key(u0, tag[a]);
            float k1 = tag_key(u1, tag[a + H]);
            if (!FAST) {
                if (jr + b >= limr[a]) k0 = kInf;
                if (jr + b >= limr[a + H]) k1 = kInf;
            }
            acc[b + a] = fminf(acc[b + a], k0);
            acc[b + a + H] = fminf(acc[b + a + H], k1);
            cmin = fmin3(cmin, k0, k1);
        }
        const int kmin = __reduce_min_sync(kFullMask, __float_as_int(cmin));
        colkey = (lane == b) ? kmin : colkey;
    }
}

template <int R>
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
    const float ulim = (float)(1.0 + 1.0 / (double)P.m);

    // cell (column j, diagonal g) is evaluated iff j - j0 < limr
    int limr[R];
    int minlim = INT32_MAX;
    unsigned tag[R];
#pragma unroll
    for (int a = 0; a < R; ++a) {
        const int64_t g = g0 + a;
        limr[a] = (g < P.g_hi) ? (int)(min(P.PL - g, j1) - j0) : 0;
        minlim = min(minlim, limr[a]);
        tag[a] = ((unsigned)lane << 3) | (unsigned)a;
    }

    // ---- FP64 re-anchor: cov(j0, j0+g) for the lane's R diagonals ----------
    double q[R];
#pragma unroll
    for (int a = 0; a < R; ++a) q[a] = 0.0;
    {
        const double* Ac = P.A + j0;
        const double* Aw = P.A + j0 + g0;
        double w[R];
#pragma unroll
        for (int a = 0; a < R - 1; ++a) w[a] = __ldg(Aw + a);
        int64_t k0 = 0;
        for (; k0 + R <= P.m; k0 += R) {
#pragma unroll
            for (int kk = 0; kk < R; ++kk) {
                w[(kk + R - 1) % R] = __ldg(Aw + k0 + kk + R - 1);
                const double x = __ldg(Ac + k0 + kk);
#pragma unroll
                for (int a = 0; a < R; ++a) q[a] = __fma_rn(x, w[(kk + a) % R], q[a]);
            }
        }
        for (int64_t k = k0; k < P.m; ++k) {
            const double x = __ldg(Ac + k);
#pragma unroll
            for (int a = 0; a < R; ++a) q[a] = __fma_rn(x, __ldg(Aw + k + a), q[a]);
        }
    }
    unsigned long long nc2[H];
    {
        const double mu0 = (double)P.m * __ldg(P.mean + j0);
        float nc[R];
#pragma unroll
        for (int a = 0; a < R; ++a) nc[a] = (float)__fma_rn(mu0, __ldg(P.mean + j0 + g0 + a), -q[a]);
#pragma unroll
        for (int a = 0; a < H; ++a) nc2[a] = f2_pack(nc[a], nc[a + H]);
    }

    // ---- ring of row partials for this tile: slot = (r - j0 - gb) mod RING --
    for (int k = lane; k < RING; k += 32) ring[k] = kInf;
    __syncwarp();

    float acc[2 * R - 1];
#pragma unroll
    for (int k = 0; k < 2 * R - 1; ++k) acc[k] = kInf;

    // row records of the band, tile-relative index t = row - (j0 + gb), staged
    // in the warp's shared-memory ring; before chunk c it holds t < fill
    const uint4* rsrc = reinterpret_cast<const uint4*>(
        reinterpret_cast<const RowRec*>(P.rowrec) + (j0 + gb));
    int fill = 33 * R + H;
    for (int i = lane; i < 2 * fill; i += 32) rec_store(rring, i >> 1, i & 1, __ldg(rsrc + i));
    __syncwarp();
    // column records, double-buffered per chunk (R records of 32 bytes each)
    const uint4* csrc = reinterpret_cast<const uint4*>(
        reinterpret_cast<const RowRec*>(P.colrec) + j0);
    if (lane < 2 * R) *reinterpret_cast<uint4*>(cring + 16 * lane) = __ldg(csrc + lane);
    __syncwarp();
    RowRec win[H];
#pragma unroll
    for (int k = 0; k < H - 1; ++k) {
        const char* p = rring + rec_off(rec_slot(lane * R + k));
        win[k].dfdg = *reinterpret_cast<const ulonglong2*>(p);
        win[k].nn = *reinterpret_cast<const unsigned long long*>(p + 16);
    }

    int cb = 0;  // column buffer holding the current chunk
    for (int64_t jc = j0; jc < j1; jc += R) {
        const int jr = (int)(jc - j0);
        // prefetch what the next chunk appends: R row records (lanes 0..2R-1)
        // and R column records (lanes 2R..4R-1), 16 bytes per lane
        uint4 next = (lane < 2 * R) ? __ldg(rsrc + 2 * fill + lane)
                                    : __ldg(csrc + 2 * (jr + R) + (lane - 2 * R));
        const char* rbase = rring + rec_off(rec_slot(jr + lane * R + H - 1));
        int colkey = 0x7fffffff;
        const char* cbuf = cring + cb * 32 * R;
        const bool fast = __all_sync(kFullMask, jr + R <= minlim);
        if (fast)
            chunk_fp32<R, true>(rbase, cbuf, win, nc2, acc, tag, limr, jr, lane, colkey);
        else
            chunk_fp32<R, false>(rbase, cbuf, win, nc2, acc, tag, limr, jr, lane, colkey);
        // column jc + lane's warp minimum (lanes 0..R-1)
        if (lane < R) {
            const unsigned bits = (unsigned)colkey;
            const float u = untag_value(bits);
            if (u < ulim) {
                const unsigned t = bits & kTagMask;
                const int64_t j = jc + lane;
                const int64_t q = j + gb + (int64_t)(t >> 3) * R + (t & 7u);
                atomicMin(P.key + j, ((unsigned long long)ord_f32(u) << 32) | (unsigned long long)q);
            }
        }
        if (lane < 2 * R) rec_store(rring, fill + (lane >> 1), lane & 1, next);
        else *reinterpret_cast<uint4*>(cring + (cb ^ 1) * 32 * R + 16 * (lane - 2 * R)) = next;
        cb ^= 1;
        fill += R;

        // lower half: rows jc + g0 + [0, R) are finished for this lane
        const int base = (int)((((jc - j0) / R) + lane) % 32) * R;
        float4* rv4 = reinterpret_cast<float4*>(ring + base);
#pragma unroll
        for (int v = 0; v < R / 4; ++v) {
            float4 t = rv4[v];
            t.x = fminf(t.x, acc[4 * v + 0]);
            t.y = fminf(t.y, acc[4 * v + 1]);
            t.z = fminf(t.z, acc[4 * v + 2]);
            t.w = fminf(t.w, acc[4 * v + 3]);
            rv4[v] = t;
        }
        __syncwarp();
        // rows jc + gb + [0, R) have met every lane of the warp
        if (lane < R) {
            const int e = (int)(((jc - j0) / R) % 32) * R + lane;
            const float v = ring[e];
            ring[e] = kInf;
            flush_row<R>(P, v, jc + gb + lane, gb, ulim);
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < R - 1; ++k) acc[k] = acc[k + R];
#pragma unroll
        for (int k = R - 1; k < 2 * R - 1; ++k) acc[k] = kInf;
    }

    // drain the rows still in flight
    const int64_t jend = j0 + ((j1 - j0 + R - 1) / R) * R;
    {
        const int base = (int)((((jend - j0) / R) + lane) % 32) * R;
#pragma unroll
        for (int k = 0; k < R - 1; ++k) ring[base + k] = fminf(ring[base + k], acc[k]);
    }
    __syncwarp();
    for (int e = lane; e < RING; e += 32) {
        const int64_t rel = ((int64_t)e - (jend - j0) % RING + RING) % RING;
        flush_row<R>(P, ring[e], jend + gb + rel, gb, ulim);
    }
    __syncwarp();
}

constexpr int kFp32WarpsPerBlock = 4;

template <int R>
constexpr int fp32_smem_bytes() {
    return kFp32WarpsPerBlock * (kRecRingBytes + 32 * R * (int)sizeof(float) + 2 * 32 * R);
}

template <int R>
__global__ void __launch_bounds__(32 * kFp32WarpsPerBlock, 4)
    fp32_tile_kernel(const Fp32TileParams P, int64_t first_tile, int64_t count) {
    extern __shared__ __align__(128) char smem_fp32[];
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;
    char* rring = smem_fp32 + w * kRecRingBytes;
    float* ring = reinterpret_cast<float*>(smem_fp32 + kFp32WarpsPerBlock * kRecRingBytes) +
                  w * 32 * R;
    char* cring = smem_fp32 + kFp32WarpsPerBlock * (kRecRingBytes + 32 * R * (int)sizeof(float)) +
                  w * 2 * 32 * R;
    const int64_t t = (int64_t)blockIdx.x * kFp32WarpsPerBlock + w;
    if (t >= count) return;
    // tile t -> band pair p, slot s; the pair's bands k and nbands-1-k have
    // nearly complementary lengths, so pairs carry nearly equal tile counts.
    // Consecutive tiles are consecutive column segments of one band: tiles
    // running together touch disjoint columns and rows.
    const int64_t tt = first_tile + t;
    const int64_t p = tt / P.seg_per_pair;
    int64_t s = tt % P.seg_per_pair;
    const int64_t span = 32 * R;
    const int64_t nseg0 = (P.PL - (P.g_lo + p * span) + P.K - 1) / P.K;
    if (s < nseg0) {
        tile_fp32<R>(P, p, s, lane, ring, rring, cring);
        return;
    }
    s -= nseg0;
    const int64_t p2 = P.nbands - 1 - p;
    if (p2 <= p) return;
    const int64_t nseg1 = (P.PL - (P.g_lo + p2 * span) + P.K - 1) / P.K;
    if (s < nseg1) tile_fp32<R>(P, p2, s, lane, ring, rring, cring);
}

}  // namespace

template <int R>
void launch_fp32_tiles(const Fp32TileParams& P, int64_t first_tile, int64_t count, cudaStream_t s) {
    const int64_t blocks = (count + kFp32WarpsPerBlock - 1) / kFp32WarpsPerBlock;
    constexpr int smem = fp32_smem_bytes<R>();
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(fp32_tile_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        configured = true;
    }
    if (blocks > 0)
        fp32_tile_kernel<R><<<(unsigned)blocks, 32 * kFp32WarpsPerBlock, smem, s>>>(P, first_tile, count);
}

template void launch_fp32_tiles<8>(const Fp32TileParams&, int64_t, int64_t, cudaStream_t);

}  // namespace mpgpu
