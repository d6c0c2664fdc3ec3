// Algorithm-variant interface of the matrix-profile engine.
//
// Mirrors the reference's plugin API so a caller written against it links
// unchanged: IMatProfAlgo {initialize, compute_matrix_profile, log_info},
// a name-keyed singleton MatProfImplFactory and static self-registration
// through FactoryRegistration<impl>("name")
// (scrimppp/inc/MatProfAlgo.hpp:15-42, scrimppp/src/MatProfAlgo.cpp:11-37),
// with the run parameters of scrimppp/inc/ScrimpppParams.hpp:6-28.
// The GPU variants registered in gpu_variants.cpp implement it on top of the
// C ABI in include/mpgpu.h.
#pragma once

#include <map>
#include <memory>
#include <string>

namespace matrix_profile {

struct Scrimppp_params {
    // fields of the reference (ScrimpppParams.hpp:6-28), same defaults
    std::string algo_name;
    std::string time_series_filename;
    std::string output_filename;
    int query_window_len;
    int prescrimp_stride;  // accepted and unused on this path, as in the reference
    int block_length;
    enum FILETYPE { BY_SUFFIX, ASCII, BIN } filetype;
    bool use_distributed_io;
    int writing_chunk_size;
    // GPU variants only
    int device;
    long reanchor_k;  // FP32 form: recurrence steps between FP64 re-anchors
    size_t mem_budget_bytes;

    Scrimppp_params()
        : algo_name(""),
          time_series_filename(""),
          output_filename("matprof"),
          query_window_len(0),
          prescrimp_stride(0),
          block_length(500),
          filetype(BY_SUFFIX),
          use_distributed_io(true),
          writing_chunk_size(0),
          device(0),
          reanchor_k(1024),
          mem_budget_bytes(0) {}
};

class IMatProfAlgo {
public:
    virtual ~IMatProfAlgo() = default;
    virtual void initialize(const Scrimppp_params& params) = 0;
    virtual void compute_matrix_profile(const Scrimppp_params& params) = 0;
    virtual void log_info() {}
};

class MatProfImplFactory {
public:
    using Creator = std::unique_ptr<IMatProfAlgo> (*)();
    static MatProfImplFactory& getInstance();
    // false (and no change) if the name is taken
    bool register_impl(const std::string& name, Creator creator_fn);
    // space-separated names, sorted
    std::string get_available_implementations() const;
    // throws std::out_of_range for an unknown name, like the reference
    std::unique_ptr<IMatProfAlgo> create(const std::string& algo_name) const;

private:
    MatProfImplFactory() = default;
    std::map<std::string, Creator> registrations_;
};

template <class Impl>
class FactoryRegistration {
public:
    explicit FactoryRegistration(const std::string& name) {
        MatProfImplFactory::getInstance().register_impl(
            name, []() { return std::unique_ptr<IMatProfAlgo>(new Impl()); });
    }
};

}  // namespace matrix_profile
