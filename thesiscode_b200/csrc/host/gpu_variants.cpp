// GPU algorithm variants registered in the reference's factory interface.
//
//   gpu_vert_blocked_fp64   drop-in for scrimp_vert_blocked
//                           (scrimppp/src/ScrimpVertBlocked.cpp:89-195): same
//                           input/output files and values, computed on the GPU
//                           with the reference's FP64 arithmetic.
//   gpu_vert_blocked_fp32k  FP32 recurrence re-anchored in FP64 every
//                           reanchor_k steps.
//
// Both read the series (ASCII or binary, ScrimpSequ.hpp:91-112), run one
// self-join through mp_selfjoin and store the profile like
// ScrimpSequ::store_matrix_profile (ScrimpSequ.cpp:253-309).
#include <chrono>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "mpgpu.h"
#include "matprof_algo.hpp"
#include "profile_io.hpp"
#include "scrimppp_merge.hpp"

namespace matrix_profile {

namespace {

// A failed library call, carrying its mp_status so that mp_run_algorithm
// returns the status itself rather than a generic one.
struct StatusError : std::runtime_error {
    StatusError(int s, const std::string& what) : std::runtime_error(what), status(s) {}
    int status;
};

std::vector<double> fetch_series(const Scrimppp_params& p) {
    switch (p.filetype) {
        case Scrimppp_params::ASCII: return io::read_series_ascii(p.time_series_filename);
        case Scrimppp_params::BIN: return io::read_series_bin(p.time_series_filename);
        default: throw std::invalid_argument("Unhandled file type detected.");
    }
}

void store_profile(const Scrimppp_params& p, const std::vector<double>& d2,
                   const std::vector<int64_t>& idx) {
    if (p.output_filename.empty()) throw std::invalid_argument("Empty output file name specified!");
    switch (p.filetype) {
        case Scrimppp_params::ASCII:
            io::write_profile_ascii(p.output_filename, d2.data(), idx.data(), (int64_t)d2.size());
            break;
        case Scrimppp_params::BIN:
            io::write_profile_bin(p.output_filename, d2.data(), idx.data(), (int64_t)d2.size());
            break;
        default: throw std::invalid_argument("Unhandled file type detected.");
    }
}

class GpuVertBlocked : public IMatProfAlgo {
public:
    explicit GpuVertBlocked(int precision) : precision_(precision) {}
    ~GpuVertBlocked() override {
        if (ctx_) mp_context_destroy(ctx_);
    }
    void initialize(const Scrimppp_params& params) override {
        if (ctx_) return;
        const int rc = mp_context_create(params.device, params.mem_budget_bytes, &ctx_);
        if (rc != MP_OK)
            throw StatusError(rc, std::string("mp_context_create: ") + mp_status_string(rc));
    }
    void compute_matrix_profile(const Scrimppp_params& params) override {
        initialize(params);
        const std::vector<double> A = fetch_series(params);
        const int64_t n = (int64_t)A.size(), m = params.query_window_len;
        if (m < 2 || n < m)
            throw std::invalid_argument(
                "ERROR: Time series is shorter than the window length, can not proceed");
        std::vector<double> d2;
        std::vector<int64_t> idx;
        join(params, A, d2, idx);
        store_profile(params, d2, idx);
    }

protected:
    mp_context* context() const { return ctx_; }

    // One self-join of A over all diagonals > m/4, with the reference's log lines.
    void join(const Scrimppp_params& params, const std::vector<double>& A, std::vector<double>& d2,
              std::vector<int64_t>& idx) {
        const int64_t n = (int64_t)A.size(), m = params.query_window_len;
        const int64_t PL = n - m + 1;
        d2.assign(PL, 0.0);
        idx.assign(PL, 0);
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = mp_selfjoin(ctx_, A.data(), n, m, -1, precision_, params.reanchor_k,
                                   params.block_length, 0, 0, d2.data(), idx.data(), nullptr);
        const double sec =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (rc != MP_OK)
            throw StatusError(rc, std::string("mp_selfjoin: ") + mp_status_string(rc) + ": " +
                                     mp_last_error(ctx_));
        const double excl = (double)(m / 4);
        const double tri = (double)PL - excl;
        std::clog << "total computation time: " << std::setprecision(17) << sec << " seconds."
                  << std::endl;
        std::clog << "throughput computations: " << tri * tri / sec << " matrix entries/second"
                  << std::endl;
        std::clog << "true cells/second: " << (tri - 1.0) * tri / 2.0 / sec << std::endl;
    }

private:
    int precision_;
    mp_context* ctx_ = nullptr;
};

class GpuVertBlockedFp64 : public GpuVertBlocked {
public:
    GpuVertBlockedFp64() : GpuVertBlocked(MP_PREC_FP64) {}
};
class GpuVertBlockedFp32K : public GpuVertBlocked {
public:
    GpuVertBlockedFp32K() : GpuVertBlocked(MP_PREC_FP32_REANCHOR) {}
};

// SCRIMP++ (ScrimpppOrig::compute_matrix_profile, scrimppp/src/ScrimpppOrig.cpp:
// 37-395): the PreSCRIMP approximate profile goes to "<output>_prescrimp"
// (always ASCII, as the reference writes it, :268-279), then the final
// profile to <output>: the exact phase (the FP64 form over all diagonals > m/4,
// the same values as scrimp_vert_blocked; the reference's own SCRIMP phase
// forms distances with sqrt-variance arithmetic, :300-330, and agrees with them
// to rounding) lowered by PreSCRIMP's neighbours exactly m/4 away, which the
// reference keeps because its exact phase never reaches them
// (merge_prescrimp_lag).
class GpuScrimppp : public GpuVertBlocked {
public:
    GpuScrimppp() : GpuVertBlocked(MP_PREC_FP64) {}
    void compute_matrix_profile(const Scrimppp_params& params) override {
        initialize(params);
        const std::vector<double> A = fetch_series(params);
        const int64_t n = (int64_t)A.size(), m = params.query_window_len;
        if (m < 2 || n < m)
            throw std::invalid_argument(
                "ERROR: Time series is shorter than the window length, can not proceed");
        const int64_t PL = n - m + 1;
        std::vector<double> d2(PL);
        std::vector<int64_t> idx(PL);
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = mp_prescrimp(context(), A.data(), n, m, (double)params.prescrimp_stride,
                                    d2.data(), idx.data(), nullptr);
        if (rc != MP_OK)
            throw StatusError(rc, std::string("mp_prescrimp: ") + mp_status_string(rc) + ": " +
                                     mp_last_error(context()));
        std::clog << "Time for PreSCRIMP: " << std::setprecision(17)
                  << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
                  << std::endl;
        if (params.output_filename.empty())
            throw std::invalid_argument("Empty output file name specified!");
        io::write_profile_ascii(params.output_filename + "_prescrimp", d2.data(), idx.data(), PL);
        std::vector<double> xd2;
        std::vector<int64_t> xidx;
        join(params, A, xd2, xidx);
        merge_prescrimp_lag(PL, m / 4, d2.data(), idx.data(), xd2.data(), xidx.data());
        store_profile(params, xd2, xidx);
    }
};

FactoryRegistration<GpuVertBlockedFp64> reg_fp64("gpu_vert_blocked_fp64");
FactoryRegistration<GpuScrimppp> reg_scrimppp("gpu_scrimppp");
FactoryRegistration<GpuVertBlockedFp32K> reg_fp32("gpu_vert_blocked_fp32k");

}  // namespace

}  // namespace matrix_profile

using matrix_profile::IMatProfAlgo;
using matrix_profile::MatProfImplFactory;
using matrix_profile::Scrimppp_params;
using matrix_profile::StatusError;
namespace io = matrix_profile::io;

extern "C" int mp_list_algorithms(char* buf, size_t len) {
    const std::string s = MatProfImplFactory::getInstance().get_available_implementations();
    if (!buf || len == 0) return (int)s.size() + 1;
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = '\0';
    return (int)s.size() + 1;
}

extern "C" int mp_run_algorithm(const char* algo, const char* input_file, const char* output_file,
                                int window_length, int prescrimp_stride, int blocklen,
                                int filetype, int64_t reanchor_k, int device) {
    if (!algo || !input_file || !output_file) return MP_ERR_INVALID_ARG;
    Scrimppp_params p;
    p.algo_name = algo;
    p.time_series_filename = input_file;
    p.output_filename = output_file;
    p.query_window_len = window_length;
    p.prescrimp_stride = prescrimp_stride;
    if (blocklen > 0) p.block_length = blocklen;
    p.filetype = filetype == 2 ? Scrimppp_params::BIN : Scrimppp_params::ASCII;
    if (reanchor_k > 0) p.reanchor_k = (long)reanchor_k;
    p.device = device;
    std::unique_ptr<IMatProfAlgo> a;
    try {
        a = MatProfImplFactory::getInstance().create(p.algo_name);
    } catch (const std::out_of_range&) {
        std::cerr << "mp_run_algorithm: unknown algorithm " << p.algo_name << std::endl;
        return MP_ERR_INVALID_ARG;
    }
    // an unreadable input is reported before any device is touched
    if (!std::ifstream(p.time_series_filename).good()) {
        std::cerr << "mp_run_algorithm: Could not open input file " << p.time_series_filename
                  << std::endl;
        return MP_ERR_IO;
    }
    try {
        a->initialize(p);
        a->compute_matrix_profile(p);
        a->log_info();
    } catch (const StatusError& e) {
        std::cerr << "mp_run_algorithm: " << e.what() << std::endl;
        return e.status;
    } catch (const io::IoError& e) {
        std::cerr << "mp_run_algorithm: " << e.what() << std::endl;
        return MP_ERR_IO;
    } catch (const std::invalid_argument& e) {
        std::cerr << "mp_run_algorithm: " << e.what() << std::endl;
        return MP_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        std::cerr << "mp_run_algorithm: " << e.what() << std::endl;
        return MP_ERR_CUDA;
    }
    return MP_OK;
}
