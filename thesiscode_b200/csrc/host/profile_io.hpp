// Series and profile files in the reference's formats.
//
// ASCII series: whitespace-separated doubles (ScrimpSequ.hpp:48-62).
// ASCII profile: one line per window, "sqrt(|d2|) index", the distance with 17
//   significant digits (ScrimpSequ.cpp:395-399).
// Binary files: a 100-byte header whose first 16 bytes are
//   {uint32 format, uint32 data_offset = 100, uint64 count} (biniobase.h:17-21),
//   zero-filled to byte 100, then the payload in native byte order:
//   format 2 = series of doubles (bintsfile.hpp:15),
//   format 1 = profile entries {double d2, uint64 index} (binproffile.h:12-16);
//   the binary profile stores the squared distance, the ASCII one its root.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace matrix_profile {
namespace io {

// A file that cannot be opened, read or written, or whose contents are not in
// the expected format.
struct IoError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

std::vector<double> read_series_ascii(const std::string& path);
std::vector<double> read_series_bin(const std::string& path);
void write_series_bin(const std::string& path, const std::vector<double>& x);
void write_profile_ascii(const std::string& path, const double* d2, const int64_t* idx, int64_t n);
void write_profile_bin(const std::string& path, const double* d2, const int64_t* idx, int64_t n);
void read_profile_bin(const std::string& path, std::vector<double>& d2, std::vector<int64_t>& idx);

}  // namespace io
}  // namespace matrix_profile
