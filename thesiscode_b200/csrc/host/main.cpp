// Command line with the reference's interface (scrimppp/src/main.cpp:176-278):
//   mpgpu_cli <algo> <window-length> <prescrimp-stride> <input-file>
//             [--blocklen B] [--output-file F] [--filetype BIN|ASCII|BY_SUFFIX]
//             [--reanchor-k K] [--device D] [--dbg] [--dist-io BOOL] [--chunksize C]
// --dbg waits for Enter before computing (a chance to attach a debugger), as in
// the reference; --dist-io and --chunksize choose how the reference's MPI ranks
// share binary file I/O: a single process writes the same bytes either way, so
// they are recorded in the parameters and change nothing here.
// The four positional arguments may also be given as --algo, --window-length,
// --prescrimp-stride, --input-file.  The file type follows the input suffix
// (.bin / .ascii) unless given; the default output name is
// <algo>_new_MatrixProfile_<m><input file name>.matprof.<ascii|bin>.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "matprof_algo.hpp"
#include "mpgpu.h"

using namespace matrix_profile;

// Boolean option values as the reference's option parser takes them.
static bool parse_bool(const std::string& v) {
    if (v == "1" || v == "true" || v == "yes" || v == "on") return true;
    if (v == "0" || v == "false" || v == "no" || v == "off") return false;
    throw std::invalid_argument("invalid boolean " + v);
}

static void usage() {
    std::cout << "usage: mpgpu_cli <algo> <window-length> <prescrimp-stride> <input-file>\n"
                 "       [--blocklen B] [--output-file F] [--filetype BIN|ASCII|BY_SUFFIX]\n"
                 "       [--reanchor-k K] [--device D] [--dbg] [--dist-io BOOL] [--chunksize C]\n"
                 "algorithms: "
              << MatProfImplFactory::getInstance().get_available_implementations() << "\n";
}

int main(int argc, char** argv) {
    Scrimppp_params p;
    p.output_filename = "";
    std::vector<std::string> pos;
    bool wait_debugger = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&](const char* name) -> std::string {
            if (i + 1 >= argc) throw std::invalid_argument(std::string("missing value for ") + name);
            return argv[++i];
        };
        try {
            if (a == "--help" || a == "-h") {
                usage();
                return 0;
            } else if (a == "--algo") pos.resize(std::max<size_t>(pos.size(), 1)), pos[0] = val("--algo");
            else if (a == "--window-length") p.query_window_len = std::stoi(val("--window-length"));
            else if (a == "--prescrimp-stride") p.prescrimp_stride = std::stoi(val("--prescrimp-stride"));
            else if (a == "--input-file") p.time_series_filename = val("--input-file");
            else if (a == "--blocklen") p.block_length = std::stoi(val("--blocklen"));
            else if (a == "--output-file") p.output_filename = val("--output-file");
            else if (a == "--reanchor-k") p.reanchor_k = std::stol(val("--reanchor-k"));
            else if (a == "--device") p.device = std::stoi(val("--device"));
            else if (a == "--dbg") wait_debugger = true;
            else if (a == "--dist-io") p.use_distributed_io = parse_bool(val("--dist-io"));
            else if (a == "--chunksize") p.writing_chunk_size = std::stoi(val("--chunksize"));
            else if (a == "--filetype") {
                const std::string t = val("--filetype");
                if (t == "BIN") p.filetype = Scrimppp_params::BIN;
                else if (t == "ASCII") p.filetype = Scrimppp_params::ASCII;
                else if (t == "BY_SUFFIX") p.filetype = Scrimppp_params::BY_SUFFIX;
                else throw std::invalid_argument("invalid filetype " + t);
            } else if (a.rfind("--", 0) == 0) {
                throw std::invalid_argument("unknown option " + a);
            } else {
                pos.push_back(a);
            }
        } catch (const std::exception& e) {
            std::cerr << "ERROR parsing commandline arguments: " << e.what() << "\n";
            usage();
            return -1;
        }
    }
    if (!pos.empty()) p.algo_name = pos[0];
    if (pos.size() > 1) p.query_window_len = std::atoi(pos[1].c_str());
    if (pos.size() > 2) p.prescrimp_stride = std::atoi(pos[2].c_str());
    if (pos.size() > 3) p.time_series_filename = pos[3];
    if (p.algo_name.empty() || p.time_series_filename.empty() || p.query_window_len == 0) {
        usage();
        return -1;
    }
    if (p.filetype == Scrimppp_params::BY_SUFFIX) {
        if (p.time_series_filename.rfind(".bin") != std::string::npos) p.filetype = Scrimppp_params::BIN;
        else if (p.time_series_filename.rfind(".ascii") != std::string::npos)
            p.filetype = Scrimppp_params::ASCII;
        else {
            std::cerr << "file type could not be determined from suffix. Specify explicitly or "
                         "rename the file...\n";
            return -1;
        }
    }
    if (p.output_filename.empty()) {
        std::string base = p.time_series_filename;
        const auto k = base.find_last_of('/');
        if (k != std::string::npos) base = base.substr(k + 1);
        p.output_filename = p.algo_name + "_new_MatrixProfile_" + std::to_string(p.query_window_len) +
                            base + ".matprof" + (p.filetype == Scrimppp_params::BIN ? ".bin" : ".ascii");
    }
    if (wait_debugger) {  // scrimppp/src/main.cpp:271-276
        std::cout << "Waiting for user input before proceeding. Chance to attach a debugger..."
                  << std::endl
                  << "Press ENTER to continue...";
        std::cout.flush();
        std::cin.get();
    }
    std::unique_ptr<IMatProfAlgo> algo;
    try {
        algo = MatProfImplFactory::getInstance().create(p.algo_name);
    } catch (const std::exception&) {
        std::cerr << "specified algorithm \"" << p.algo_name << "\" is not known. Valid algorithms: "
                  << MatProfImplFactory::getInstance().get_available_implementations() << "\n";
        return -1;
    }
    try {
        algo->initialize(p);
        algo->compute_matrix_profile(p);
        algo->log_info();
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
