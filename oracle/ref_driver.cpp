/*
 * Driver around the reference's own SCRIMP hot path (test infrastructure).
 *
 * The reference translation units (scrimppp/src/kernels.cpp, ScrimpSequ.cpp,
 * ScrimpSequOpt.cpp, ScrimpVertBlocked.cpp, MatProfAlgo.cpp, logging.cpp,
 * timing.cpp, partitioning_1d.cpp) are compiled unchanged where they lie, by
 * oracle/Makefile, against the stub headers in oracle/stubs/.  This file adds
 * no arithmetic of its own: it only feeds in-memory arrays to the reference's
 * functions in the order its drivers use them, so tests and the CPU baseline
 * can call them without files or MPI.
 *
 * Exposed entry points (extern "C"):
 *   ref_window_stats       -> ScrimpSequOpt::precompute_window_statistics
 *                             (scrimppp/src/ScrimpSequOpt.cpp:33-79)
 *   ref_first_qt           -> ScrimpSequOpt::init_diagonals (:81-96)
 *   ref_eval_diag_block_triangle -> matrix_profile::eval_diag_block_triangle
 *                             (scrimppp/inc/kernels.h:7-24, src/kernels.cpp:368-410)
 *   ref_vert_blocked       -> the body of ScrimpVertBlocked::compute_matrix_profile
 *                             (scrimppp/src/ScrimpVertBlocked.cpp:89-174) minus file I/O
 *   ref_triv_par_threads   -> ScrimpTrivialPar's diagonal partitioning
 *                             (scrimppp/src/ScrimpTrivialPar.cpp:200-340), re-hosted
 *                             on std::thread instead of MPI ranks, merged on the
 *                             host with the min-by-distance rule of its MPI_Op
 *                             (:68-108).
 * and a command-line front end with the reference's positional arguments
 * (algo, window length, PreSCRIMP stride, input file) that runs the
 * reference's own factory + compute_matrix_profile path on ASCII files.
 */
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include <MatProfAlgo.hpp>
#include <ScrimpVertBlocked.hpp>
#include <kernels.h>
#include <partitioning_1d.h>

namespace matrix_profile {

/* Makes the protected helpers of the reference classes callable. */
class RefAccess : public ScrimpVertBlocked {
public:
    static void stats(int m, const aligned_tsdtype_vec& A, int PL, aligned_tsdtype_vec& muS,
                      aligned_tsdtype_vec& sInv) {
        ScrimpSequOpt::precompute_window_statistics(m, A, PL, muS, sInv);
    }
    void init_diags(int first, int last, aligned_tsdtype_vec& qt, const aligned_tsdtype_vec& A,
                    int m) {
        init_diagonals(first, last, qt, A, m);
    }
    void eval_block(int B, aligned_int_vec& idx, const aligned_tsdtype_vec& A,
                    aligned_tsdtype_vec& qt, int m, const aligned_tsdtype_vec& sInv,
                    const aligned_tsdtype_vec& muS, int d0, aligned_tsdtype_vec& prof) {
        eval_diagonal_block(B, idx, A, qt, m, sInv, muS, d0, prof);
    }
};

}  // namespace matrix_profile

using namespace matrix_profile;

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

extern "C" {

int ref_window_stats(const double* A, long n, long m, double* muS_out, double* sInv_out) {
    if (m < 2 || n < m) return -1;
    aligned_tsdtype_vec a(A, A + n), muS(n), sInv(n);
    const long PL = n - m + 1;
    RefAccess::stats((int)m, a, (int)PL, muS, sInv);
    std::memcpy(muS_out, muS.data(), PL * sizeof(double));
    std::memcpy(sInv_out, sInv.data(), PL * sizeof(double));
    return 0;
}

/* First dot product of each diagonal d in [first, last] (inclusive, like the
 * reference), written to qt_out[d - first].  last must be <= n - m so no read
 * goes past the series (the reference's init_all_diagonals also evaluates
 * d = n - m + 1, one element past the end; that diagonal is never used). */
int ref_first_qt(const double* A, long n, long m, long first, long last, double* qt_out) {
    if (m < 1 || n < m || first < 0 || last > n - m || last < first) return -1;
    aligned_tsdtype_vec a(A, A + n), qt(n);
    RefAccess acc;
    acc.init_diags((int)first, (int)last, qt, a, (int)m);
    std::memcpy(qt_out, qt.data() + first, (last - first + 1) * sizeof(double));
    return 0;
}

void ref_eval_diag_block_triangle(double* prof_colmin, long* idx_colmin, double* prof_rowmin,
                                  long* idx_rowmin, double* tmpQ, long blocklen, long trianglen,
                                  const double* A_hor, const double* A_vert, long m,
                                  const double* s_hor, const double* mu_hor, const double* s_vert,
                                  const double* mu_vert, long baserow, long basecol) {
    eval_diag_block_triangle(prof_colmin, idx_colmin, prof_rowmin, idx_rowmin, tmpQ, blocklen,
                             trianglen, A_hor, A_vert, m, s_hor, mu_hor, s_vert, mu_vert, baserow,
                             basecol);
}

/* ScrimpVertBlocked::compute_matrix_profile (ScrimpVertBlocked.cpp:93-174)
 * without the file read/write: same statistics, same first-QT init, same block
 * list excl+1, excl+1+B, ... <= PL, optionally shuffled with the same
 * std::random_shuffle, the same per-block kernel call and the same score ->
 * squared-distance transform.  d2_out/idx_out receive PL entries. */
int ref_vert_blocked(const double* A, long n, long m, long blocklen, int shuffle, double* d2_out,
                     long* idx_out, double* seconds) {
    if (m < 2 || n < m || blocklen < 1) return -1;
    aligned_tsdtype_vec a(A, A + n);
    aligned_tsdtype_vec muS(n), sInv(n);
    const int windowSize = (int)m;
    const int exclusionZone = windowSize / 4;
    const int PL = (int)(n - m + 1);
    aligned_tsdtype_vec profile(PL, -1.0);
    aligned_int_vec profileIndex(PL, 0);
    aligned_tsdtype_vec initial_zs(n);
    std::vector<int> idx;
    RefAccess acc;
    const double t0 = now_s();
    RefAccess::stats(windowSize, a, PL, muS, sInv);
    if (PL - 1 >= 0) acc.init_diags(0, PL - 1, initial_zs, a, windowSize);
    for (int i = exclusionZone + 1; i <= PL; i += (int)blocklen) idx.push_back(i);
    if (shuffle) std::random_shuffle(idx.begin(), idx.end());
    for (size_t ri = 0; ri < idx.size(); ++ri)
        acc.eval_block((int)blocklen, profileIndex, a, initial_zs, windowSize, sInv, muS, idx[ri],
                       profile);
    const double twice_m = 2.0 * static_cast<double>(windowSize);
    for (auto it = profile.begin(); it < profile.end(); ++it) *it = twice_m - 2.0 * (*it);
    if (seconds) *seconds = now_s() - t0;
    std::memcpy(d2_out, profile.data(), PL * sizeof(double));
    std::memcpy(idx_out, profileIndex.data(), PL * sizeof(long));
    return 0;
}

/* ScrimpTrivialPar's work split (ScrimpTrivialPar.cpp:200-224, 270-298) run
 * by nthreads threads instead of MPI ranks, restricted to the diagonal range
 * [diag_lo, diag_hi) (diag_lo >= excl+1, diag_hi <= PL).  Rank r takes
 * partitions r and 2P-1-r of that range (partitioning_1d.cpp:8-31), splits
 * each into blocks of at most blocklen diagonals, inits their first dot
 * products and calls the reference kernel per block on its private result
 * (profile -1, index -1, :167-168).  Scores go to squared distances
 * (:336-340, without the one-past-end write) and the rank results are merged
 * in rank order with the strict min-by-distance rule of the reference's
 * reduction op (:100-107).  seconds receives the wall time of everything
 * after argument checks. */
int ref_triv_par_threads(const double* A, long n, long m, long blocklen, long diag_lo,
                         long diag_hi, int nthreads, double* d2_out, long* idx_out,
                         double* seconds) {
    if (m < 2 || n < m || blocklen < 1 || nthreads < 1) return -1;
    const long PL = n - m + 1;
    const long excl = m / 4;
    if (diag_lo < excl + 1 || diag_hi > PL || diag_hi <= diag_lo) return -2;
    aligned_tsdtype_vec a(A, A + n);
    aligned_tsdtype_vec muS(n), sInv(n);
    const double t0 = now_s();
    RefAccess::stats((int)m, a, (int)PL, muS, sInv);

    const int P = nthreads;
    const int ndiag = (int)(diag_hi - diag_lo);
    const PartitioningInfo info = split_work(2 * P, ndiag);
    std::vector<aligned_tsdtype_vec> prof(P);
    std::vector<aligned_int_vec> pidx(P);
    std::vector<std::thread> pool;
    for (int r = 0; r < P; ++r) {
        pool.emplace_back([&, r]() {
            prof[r].assign(PL, -1.0);
            pidx[r].assign(PL, -1);
            aligned_tsdtype_vec qt(n);
            RefAccess acc;
            for (int half = 0; half < 2; ++half) {
                const int part_id = half == 0 ? r : 2 * P - 1 - r;
                if (get_workload(part_id, info) <= 0) continue;
                const Partition1D part = get_partition(part_id, info);
                const int first = (int)diag_lo + part._first_id;
                const int last = std::min((int)diag_hi - 1, (int)diag_lo + part._last_id);
                for (int b0 = first; b0 <= last; b0 += (int)blocklen) {
                    const int b1 = std::min(b0 + (int)blocklen - 1, last);
                    acc.init_diags(b0, b1, qt, a, (int)m);
                    eval_diag_block_triangle(prof[r].data(), pidx[r].data(), prof[r].data() + b0,
                                             pidx[r].data() + b0, qt.data() + b0, b1 - b0 + 1,
                                             PL - b0, a.data(), a.data() + b0, m, sInv.data(),
                                             muS.data(), sInv.data() + b0, muS.data() + b0, b0, 0);
                }
            }
            const double twice_m = 2.0 * static_cast<double>(m);
            for (long i = 0; i < PL; ++i) prof[r][i] = twice_m - 2.0 * prof[r][i];
        });
    }
    for (auto& t : pool) t.join();
    for (long i = 0; i < PL; ++i) {
        double best = prof[0][i];
        long bi = pidx[0][i];
        for (int r = 1; r < P; ++r)
            if (prof[r][i] < best) {
                best = prof[r][i];
                bi = pidx[r][i];
            }
        d2_out[i] = best;
        idx_out[i] = bi;
    }
    if (seconds) *seconds = now_s() - t0;
    return 0;
}

}  // extern "C"

/* Command line: <algo> <window-length> <prescrimp-stride> <input-file>
 *               [--blocklen B] [--output-file F] [--filetype ASCII|BIN]
 * Runs the reference's factory + compute_matrix_profile on an ASCII series,
 * the same calls its main() makes (scrimppp/src/main.cpp:47-80). */
int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr,
                     "usage: %s <algo> <window-length> <prescrimp-stride> <input-file> "
                     "[--blocklen B] [--output-file F] [--filetype ASCII|BIN]\navailable: %s\n",
                     argv[0], MatProfImplFactory::getInstance().get_available_implementations().c_str());
        return 2;
    }
    Scrimppp_params p;
    p.algo_name = argv[1];
    p.query_window_len = std::atoi(argv[2]);
    p.prescrimp_stride = std::atoi(argv[3]);
    p.time_series_filename = argv[4];
    p.filetype = Scrimppp_params::ASCII;
    p.output_filename = "";
    for (int i = 5; i + 1 < argc; i += 2) {
        std::string k = argv[i];
        if (k == "--blocklen") p.block_length = std::atoi(argv[i + 1]);
        else if (k == "--filetype")  // BIN needs the reference's MPI-IO classes (scrimppp_ref_bin)
            p.filetype = std::string(argv[i + 1]) == "BIN" ? Scrimppp_params::BIN
                                                          : Scrimppp_params::ASCII;
        else if (k == "--output-file") p.output_filename = argv[i + 1];
    }
    if (p.output_filename.empty()) {
        std::string base = p.time_series_filename;
        std::string::size_type k = base.find_last_of('/');
        if (k != std::string::npos) base = base.substr(k + 1);
        p.output_filename = p.algo_name + "_new_MatrixProfile_" + std::to_string(p.query_window_len) +
                            base + ".matprof.ascii";
    }
    std::unique_ptr<IMatProfAlgo> algo;
    try {
        algo = MatProfImplFactory::getInstance().create(p.algo_name);
    } catch (const std::exception&) {
        std::fprintf(stderr, "unknown algorithm %s\n", p.algo_name.c_str());
        return 1;
    }
    algo->initialize(p);
    algo->compute_matrix_profile(p);
    return 0;
}
