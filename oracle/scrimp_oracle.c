/*
 * CPU oracle for the diagonal-blocked SCRIMP self-join -- TEST INFRASTRUCTURE.
 *
 * Plain-C restatement of the reference's hot path.  Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load it, and only as the checker.
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off: every product and sum is
 * rounded where the source writes it; fma() is the explicit fused op the
 * reference's AVX2 intrinsics perform).
 *
 * Parity pin: tests/test_oracle.py compares each function bit-for-bit with the
 * reference's own sources compiled unchanged (oracle/_ref, IEEE build) and with
 * the golden vectors under tests/golden/ that the reference produced.
 */
#include "scrimp_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

/* scrimppp/src/ScrimpSequOpt.cpp:33-79: prefix sums of x and x^2 in index
 * order, window sums as differences of prefix sums, mean = S/m,
 * var = S2/m - mean^2, sInv = 1/sqrt(var), muS = (mean*sInv)*sqrt(m). */
int orc_window_stats(const double* A, int64_t n, int64_t m, double* muS, double* sInv) {
    if (m < 1 || n < m) return -1;
    const int64_t PL = n - m + 1;
    const double dm = (double)m;
    const double sqrt_m = sqrt(dm);
    double* cs = (double*)malloc(sizeof(double) * n);
    double* cs2 = (double*)malloc(sizeof(double) * n);
    if (!cs || !cs2) {
        free(cs);
        free(cs2);
        return -2;
    }
    cs[0] = A[0];
    for (int64_t i = 1; i < n; ++i) cs[i] = A[i] + cs[i - 1];
    cs2[0] = A[0] * A[0];
    for (int64_t i = 1; i < n; ++i) cs2[i] = A[i] * A[i] + cs2[i - 1];
    for (int64_t i = 0; i < PL; ++i) {
        const double s = (i == 0) ? cs[m - 1] : cs[m - 1 + i] - cs[i - 1];
        const double s2 = (i == 0) ? cs2[m - 1] : cs2[m - 1 + i] - cs2[i - 1];
        const double mean = s / dm;
        const double var = s2 / dm - mean * mean;
        const double si = 1.0 / sqrt(var);
        sInv[i] = si;
        muS[i] = mean * si * sqrt_m;
    }
    free(cs);
    free(cs2);
    return 0;
}

/* ScrimpSequOpt.cpp:81-96: lastz += A[k+diag]*A[k] for k = 0..m-1. */
int orc_first_qt(const double* A, int64_t n, int64_t m, int64_t d_lo, int64_t d_hi, double* qt) {
    if (m < 1 || n < m || d_lo < 0 || d_hi > n - m + 1 || d_hi < d_lo) return -1;
    for (int64_t d = d_lo; d < d_hi; ++d) {
        double z = 0.0;
        for (int64_t k = 0; k < m; ++k) z += A[k + d] * A[k];
        qt[d - d_lo] = z;
    }
    return 0;
}

/* Core of the block kernel (scrimppp/src/kernels.cpp:170-307), evaluating
 * only diagonals whose offset in the block lies in [dlo, dhi).  The
 * vector/remainder split -- which decides whether a cell uses the fused
 * (FMA) or the separately rounded arithmetic -- depends on the full block
 * (blocklen, trianglen) exactly as in the reference, so a restricted call
 * computes every evaluated cell bit-identically to a full call. */
static void block_core(double* prof_col, int64_t* idx_col, double* prof_row, int64_t* idx_row,
                       double* tmpQ, int64_t blocklen, int64_t trianglen, const double* A_hor,
                       const double* A_vert, int64_t m, const double* s_hor, const double* mu_hor,
                       const double* s_vert, const double* mu_vert, int64_t baserow,
                       int64_t basecol, int64_t dlo, int64_t dhi) {
    for (int64_t j = 0; j < trianglen; ++j) {
        const int64_t cnt = blocklen < trianglen - j ? blocklen : trianglen - j;
        const int64_t nvec = cnt - cnt % 4; /* 4-wide part, kernels.cpp:194-197 */
        const double sh = s_hor[j], mh = mu_hor[j], ah = A_hor[j], ahf = A_hor[j + m];
        const int64_t col_in_mat = j + basecol;
        /* per-lane running best of the column, seeded with the stored value */
        double lane_best[4];
        int64_t lane_idx[4];
        for (int l = 0; l < 4; ++l) {
            lane_best[l] = prof_col[j];
            lane_idx[l] = idx_col[j] + l; /* lane offset added before the reduction, :251-253 */
        }
        int64_t v = 0;
        for (; v < nvec; v += 4) {
            for (int l = 0; l < 4; ++l) {
                const int64_t dg = v + l;
                if (dg < dlo || dg >= dhi) continue;
                const int64_t i = j + dg;
                /* score = QT*(s_v*s_h) - mu_h*mu_v with one rounding, :206-215 */
                const double ss = s_vert[i] * sh;
                const double mm = mh * mu_vert[i];
                const double score = fma(tmpQ[dg], ss, -mm);
                /* QT += A_v[i+m]*A_h[j+m] (fused), QT -= A_v[i]*A_h[j] (fused), :218-225 */
                double q = fma(A_vert[i + m], ahf, tmpQ[dg]);
                q = fma(-A_vert[i], ah, q);
                tmpQ[dg] = q;
                if (score > prof_row[i]) { /* row side, :228-234 */
                    prof_row[i] = score;
                    idx_row[i] = col_in_mat;
                }
                if (score > lane_best[l]) { /* column side, per lane, :240-244 */
                    lane_best[l] = score;
                    lane_idx[l] = j + v + l;
                }
            }
        }
        /* lane reduction :255-278: (0,1) and (2,3) first, then (0,2); the
         * higher lane replaces the lower only if strictly greater */
        double b01 = lane_best[0];
        int64_t i01 = lane_idx[0];
        if (lane_best[1] > b01) {
            b01 = lane_best[1];
            i01 = lane_idx[1];
        }
        double b23 = lane_best[2];
        int64_t i23 = lane_idx[2];
        if (lane_best[3] > b23) {
            b23 = lane_best[3];
            i23 = lane_idx[3];
        }
        double profile_j = b01;
        int64_t index_j = i01;
        if (b23 > profile_j) {
            profile_j = b23;
            index_j = i23;
        }
        index_j += baserow;
        /* scalar remainder :282-300, each product and sum rounded separately */
        for (; v < cnt; ++v) {
            const int64_t dg = v;
            if (dg < dlo || dg >= dhi) continue;
            const int64_t i = j + dg;
            const double ss = s_vert[i] * sh;
            const double t1 = tmpQ[dg] * ss;
            const double t2 = mu_vert[i] * mh;
            const double score = t1 - t2;
            const double far = A_vert[i + m] * A_hor[j + m];
            double q = tmpQ[dg] + far;
            const double near = A_vert[i] * A_hor[j];
            q = q - near;
            tmpQ[dg] = q;
            if (score > prof_row[i]) {
                prof_row[i] = score;
                idx_row[i] = col_in_mat;
            }
            if (score > profile_j) {
                profile_j = score;
                index_j = i + baserow;
            }
        }
        if (profile_j > prof_col[j]) { /* :302-305 */
            prof_col[j] = profile_j;
            idx_col[j] = index_j;
        }
    }
}

void orc_eval_diag_block_triangle(double* prof_colmin, int64_t* idx_colmin, double* prof_rowmin,
                                  int64_t* idx_rowmin, double* tmpQ, int64_t blocklen,
                                  int64_t trianglen, const double* A_hor, const double* A_vert,
                                  int64_t m, const double* s_hor, const double* mu_hor,
                                  const double* s_vert, const double* mu_vert, int64_t baserow,
                                  int64_t basecol) {
    block_core(prof_colmin, idx_colmin, prof_rowmin, idx_rowmin, tmpQ, blocklen, trianglen, A_hor,
               A_vert, m, s_hor, mu_hor, s_vert, mu_vert, baserow, basecol, 0, blocklen);
}

typedef struct {
    const double* A;
    int64_t n, m, PL, excl, B, lo, hi, nblocks;
    const double* muS;
    const double* sInv;
    atomic_long next;
    double** prof;
    int64_t** idx;
    int status;
} join_job;

typedef struct {
    join_job* job;
    int tid;
} join_arg;

static void* join_worker(void* p) {
    join_arg* a = (join_arg*)p;
    join_job* jb = a->job;
    double* prof = jb->prof[a->tid];
    int64_t* idx = jb->idx[a->tid];
    double* qt = (double*)malloc(sizeof(double) * (jb->B > 0 ? jb->B : 1));
    if (!qt) {
        jb->status = -2;
        return NULL;
    }
    for (;;) {
        const long k = atomic_fetch_add(&jb->next, 1);
        if (k >= jb->nblocks) break;
        const int64_t b0 = jb->excl + 1 + k * jb->B;
        const int64_t lo = jb->lo > b0 ? jb->lo : b0;
        const int64_t hi = jb->hi < b0 + jb->B ? jb->hi : b0 + jb->B;
        if (hi <= lo) continue;
        /* the first dot products of the evaluated diagonals (others unused) */
        orc_first_qt(jb->A, jb->n, jb->m, lo, hi, qt + (lo - b0));
        block_core(prof, idx, prof + b0, idx + b0, qt, jb->B, jb->PL - b0, jb->A, jb->A + b0,
                   jb->m, jb->sInv, jb->muS, jb->sInv + b0, jb->muS + b0, b0, 0, lo - b0,
                   hi - b0);
    }
    free(qt);
    return NULL;
}

int orc_selfjoin_fp64(const double* A, int64_t n, int64_t m, int64_t excl, int64_t blocklen,
                      int64_t diag_lo, int64_t diag_hi, int nthreads, double* d2, int64_t* idx) {
    if (m < 2 || n < m || blocklen < 1) return -1;
    const int64_t PL = n - m + 1;
    if (excl < 0) excl = m / 4;
    if (diag_lo == 0 && diag_hi == 0) {
        diag_lo = excl + 1;
        diag_hi = PL;
    }
    if (diag_lo < excl + 1) diag_lo = excl + 1;
    if (diag_hi > PL) diag_hi = PL;
    if (nthreads < 1) nthreads = 1;
    double* muS = (double*)malloc(sizeof(double) * PL);
    double* sInv = (double*)malloc(sizeof(double) * PL);
    if (!muS || !sInv) {
        free(muS);
        free(sInv);
        return -2;
    }
    orc_window_stats(A, n, m, muS, sInv);
    join_job jb;
    jb.A = A;
    jb.n = n;
    jb.m = m;
    jb.PL = PL;
    jb.excl = excl;
    jb.B = blocklen;
    jb.lo = diag_lo;
    jb.hi = diag_hi;
    jb.nblocks = (PL - excl - 1 + blocklen - 1) / blocklen; /* blocks excl+1 + k*B < PL */
    if (jb.nblocks < 0) jb.nblocks = 0;
    jb.muS = muS;
    jb.sInv = sInv;
    atomic_init(&jb.next, 0);
    jb.status = 0;
    jb.prof = (double**)calloc(nthreads, sizeof(double*));
    jb.idx = (int64_t**)calloc(nthreads, sizeof(int64_t*));
    int rc = 0;
    for (int t = 0; t < nthreads; ++t) {
        jb.prof[t] = (t == 0) ? d2 : (double*)malloc(sizeof(double) * PL);
        jb.idx[t] = (t == 0) ? idx : (int64_t*)malloc(sizeof(int64_t) * PL);
        if (!jb.prof[t] || !jb.idx[t]) rc = -2;
    }
    if (rc == 0) {
        for (int t = 0; t < nthreads; ++t)
            for (int64_t i = 0; i < PL; ++i) {
                jb.prof[t][i] = -1.0; /* ScrimpVertBlocked.cpp:103-104 */
                jb.idx[t][i] = 0;
            }
        pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
        join_arg* args = (join_arg*)malloc(sizeof(join_arg) * nthreads);
        for (int t = 0; t < nthreads; ++t) {
            args[t].job = &jb;
            args[t].tid = t;
            if (t > 0) pthread_create(&th[t], NULL, join_worker, &args[t]);
        }
        join_worker(&args[0]);
        for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
        free(th);
        free(args);
        rc = jb.status;
        for (int t = 1; t < nthreads; ++t)
            for (int64_t i = 0; i < PL; ++i)
                if (jb.prof[t][i] > d2[i]) {
                    d2[i] = jb.prof[t][i];
                    idx[i] = jb.idx[t][i];
                }
        /* ScrimpVertBlocked.cpp:171-174 */
        const double twice_m = 2.0 * (double)m;
        for (int64_t i = 0; i < PL; ++i) d2[i] = twice_m - 2.0 * d2[i];
    }
    for (int t = 1; t < nthreads; ++t) {
        free(jb.prof[t]);
        free(jb.idx[t]);
    }
    free(jb.prof);
    free(jb.idx);
    free(muS);
    free(sInv);
    return rc;
}

/* One cell's score in the reference's arithmetic: the diagonal g = row - col
 * runs from its first dot product (ScrimpSequOpt.cpp:81-96) through the block
 * of blocklen diagonals that holds it (ScrimpVertBlocked.cpp:139-142: cut at
 * excl+1 + k*blocklen, triangle length PL - block start), each cell fused or
 * separately rounded as its position in that block selects -- the same
 * per-cell operations as block_core above (kernels.cpp:194-300). */
int orc_cell_scores(const double* A, int64_t n, int64_t m, int64_t excl, int64_t blocklen,
                    const double* muS, const double* sInv, int64_t count, const int64_t* col,
                    const int64_t* row, double* score) {
    if (m < 2 || n < m || blocklen < 1) return -1;
    const int64_t PL = n - m + 1;
    if (excl < 0) excl = m / 4;
    for (int64_t k = 0; k < count; ++k) {
        const int64_t c = col[k], r = row[k], g = r - c;
        if (c < 0 || r >= PL || g < excl + 1) return -2;
        const int64_t d0 = excl + 1 + ((g - excl - 1) / blocklen) * blocklen;
        const int64_t dg = g - d0, T = PL - d0;
        double q;
        orc_first_qt(A, n, m, g, g + 1, &q);
        double sc = NAN;
        for (int64_t j = 0; j <= c; ++j) {
            const int64_t cnt = blocklen < T - j ? blocklen : T - j;
            const int64_t nvec = cnt - cnt % 4;
            const double sh = sInv[j], mh = muS[j], sv = sInv[j + g], mv = muS[j + g];
            if (dg < nvec) {
                const double ss = sv * sh;
                const double mm = mh * mv;
                sc = fma(q, ss, -mm);
                double t = fma(A[j + g + m], A[j + m], q);
                q = fma(-A[j + g], A[j], t);
            } else {
                const double ss = sv * sh;
                const double t1 = q * ss;
                const double t2 = mv * mh;
                sc = t1 - t2;
                const double far = A[j + g + m] * A[j + m];
                double t = q + far;
                const double near = A[j + g] * A[j];
                q = t - near;
            }
        }
        score[k] = sc;
    }
    return 0;
}

double orc_pair_d2(const double* A, int64_t n, int64_t m, int64_t i, int64_t j) {
    if (i < 0 || j < 0 || i + m > n || j + m > n) return NAN;
    long double si = 0, sj = 0;
    for (int64_t k = 0; k < m; ++k) {
        si += A[i + k];
        sj += A[j + k];
    }
    const long double mi = si / m, mj = sj / m;
    long double vi = 0, vj = 0, c = 0;
    for (int64_t k = 0; k < m; ++k) {
        const long double a = A[i + k] - mi, b = A[j + k] - mj;
        vi += a * a;
        vj += b * b;
        c += a * b;
    }
    if (vi == 0 || vj == 0) return NAN;
    const long double rho = c / sqrtl(vi * vj);
    return (double)(2.0L * m * (1.0L - rho));
}

double orc_cells(int64_t n, int64_t m, int64_t diag_lo, int64_t diag_hi) {
    const int64_t PL = n - m + 1;
    double cells = 0;
    for (int64_t d = diag_lo; d < diag_hi; ++d)
        if (d > 0 && d < PL) cells += (double)(PL - d);
    return cells;
}
