/*
 * CPU oracle for the diagonal-blocked SCRIMP self-join -- TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference's hot path, evaluated with IEEE
 * double arithmetic in the reference's own operation order.  Only tests, the
 * smoke check and the CPU-baseline leg of bench.py use it, and only as the
 * checker; the product library never calls it.
 *
 * Parity pin: tests/test_oracle.py checks every function here bit-for-bit
 * against the reference's own sources compiled unchanged (oracle/_ref, IEEE
 * build) and against the golden vectors in tests/golden/ that those sources
 * produced.
 */
#ifndef SCRIMP_ORACLE_H
#define SCRIMP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Window statistics, scrimppp/src/ScrimpSequOpt.cpp:33-79.
 * muS[i] = mean_i * sInv_i * sqrt(m), sInv[i] = 1/sqrt(var_i), i < n-m+1. */
int orc_window_stats(const double* A, int64_t n, int64_t m, double* muS, double* sInv);

/* First dot product of diagonals d in [d_lo, d_hi), ScrimpSequOpt.cpp:81-96:
 * qt[d - d_lo] = sum_{k<m} A[k+d]*A[k], summed in k order. */
int orc_first_qt(const double* A, int64_t n, int64_t m, int64_t d_lo, int64_t d_hi, double* qt);

/* One block of diagonals, same arguments and semantics as the reference's
 * eval_diag_block_triangle (scrimppp/inc/kernels.h:7-24), arithmetic of its
 * AVX2 branch (scrimppp/src/kernels.cpp:170-307) including the 4-lane column
 * reduction and the scalar remainder. */
void orc_eval_diag_block_triangle(double* prof_colmin, int64_t* idx_colmin, double* prof_rowmin,
                                  int64_t* idx_rowmin, double* tmpQ, int64_t blocklen,
                                  int64_t trianglen, const double* A_hor, const double* A_vert,
                                  int64_t m, const double* s_hor, const double* mu_hor,
                                  const double* s_vert, const double* mu_vert, int64_t baserow,
                                  int64_t basecol);

/* Whole self-join restricted to diagonals [diag_lo, diag_hi) (pass 0,0 for
 * the full range excl+1 .. PL-1), ScrimpVertBlocked.cpp:89-174 with the block
 * list in natural order.  Blocks are cut at excl+1 + k*blocklen as in the
 * reference (a restricted range uses the same cut points).  excl < 0 selects
 * m/4.  Outputs PL = n-m+1 squared distances (2m - 2*score) and indices;
 * windows that no cell improved keep score -1 (d2 = 2m+2) and index 0.
 * nthreads > 1 splits the block list across threads; per-thread results are
 * merged in thread order with the strict '>' of the reference (values are
 * identical for any split; only exact-tie indices can move). */
int orc_selfjoin_fp64(const double* A, int64_t n, int64_t m, int64_t excl, int64_t blocklen,
                      int64_t diag_lo, int64_t diag_hi, int nthreads, double* d2, int64_t* idx);

/* Scores that the reference's arithmetic gives the cells (col[k], row[k]),
 * col < row, row - col > excl, in a vert_blocked join with this blocklen:
 * the cell's diagonal is run from its first dot product with the fused or
 * separately rounded operations its place in its block selects.  muS/sInv
 * from orc_window_stats.  Cost O(col[k]) per cell.  Used to judge whether two
 * candidate neighbours tie in the reference's own values. */
int orc_cell_scores(const double* A, int64_t n, int64_t m, int64_t excl, int64_t blocklen,
                    const double* muS, const double* sInv, int64_t count, const int64_t* col,
                    const int64_t* row, double* score);

/* Squared z-normalised distance between windows i and j, evaluated in long
 * double with per-window centring (an accuracy yardstick, not the reference
 * arithmetic).  Returns NaN for a window of zero variance. */
double orc_pair_d2(const double* A, int64_t n, int64_t m, int64_t i, int64_t j);

/* Number of distance-matrix cells on diagonals [diag_lo, diag_hi). */
double orc_cells(int64_t n, int64_t m, int64_t diag_lo, int64_t diag_hi);

#ifdef __cplusplus
}
#endif

#endif
