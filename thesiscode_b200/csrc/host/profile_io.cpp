// Reader/writer for the reference's ASCII and binary series/profile files
// (formats described in profile_io.hpp).
#include "profile_io.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <stdexcept>

namespace matrix_profile {
namespace io {

namespace {

constexpr uint32_t kHeaderBytes = 100;
constexpr uint32_t kFmtProfile = 1;
constexpr uint32_t kFmtSeries = 2;

struct Header {
    uint32_t fmt;
    uint32_t data_offset;
    uint64_t count;
};
static_assert(sizeof(Header) == 16, "binary header prefix is 16 bytes");

void write_header(std::ofstream& f, uint32_t fmt, uint64_t count) {
    char buf[kHeaderBytes];
    std::memset(buf, 0, sizeof buf);
    Header h{fmt, kHeaderBytes, count};
    std::memcpy(buf, &h, sizeof h);
    f.write(buf, sizeof buf);
}

Header read_header(std::ifstream& f, uint32_t want_fmt, const std::string& path) {
    Header h{};
    f.read(reinterpret_cast<char*>(&h), sizeof h);
    if (!f) throw IoError("cannot read binary header of " + path);
    if (h.fmt != want_fmt)
        throw IoError("unexpected binary format " + std::to_string(h.fmt) + " in " + path);
    if (h.data_offset != kHeaderBytes)
        throw IoError("unexpected data offset in " + path);
    f.seekg(h.data_offset, std::ios::beg);
    return h;
}

// Payload elements of `width` bytes the file holds after the read position, so
// that a header count is checked against the file before anything is allocated.
uint64_t payload_elements(std::ifstream& f, uint64_t width) {
    const std::streampos here = f.tellg();
    f.seekg(0, std::ios::end);
    const std::streampos end = f.tellg();
    f.seekg(here);
    return end > here ? (uint64_t)(end - here) / width : 0;
}

void check_count(std::ifstream& f, const Header& h, uint64_t width, const char* what,
                 const std::string& path) {
    const uint64_t have = payload_elements(f, width);
    if (h.count > have)
        throw IoError(std::string("truncated ") + what + " file " + path + ": header says " +
                                 std::to_string(h.count) + " entries, the file holds " +
                                 std::to_string(have));
}

}  // namespace

std::vector<double> read_series_ascii(const std::string& path) {
    std::ifstream f(path);
    if (!f.is_open()) throw IoError("Could not open input file " + path);
    std::vector<double> x;
    double v;
    while (f >> v) x.push_back(v);
    return x;
}

std::vector<double> read_series_bin(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) throw IoError("Could not open input file " + path);
    const Header h = read_header(f, kFmtSeries, path);
    check_count(f, h, sizeof(double), "series", path);
    std::vector<double> x(h.count);
    f.read(reinterpret_cast<char*>(x.data()), sizeof(double) * h.count);
    if (!f) throw IoError("truncated series file " + path);
    return x;
}

void write_series_bin(const std::string& path, const std::vector<double>& x) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.is_open()) throw IoError("cannot create " + path);
    write_header(f, kFmtSeries, x.size());
    f.write(reinterpret_cast<const char*>(x.data()), sizeof(double) * x.size());
}

void write_profile_ascii(const std::string& path, const double* d2, const int64_t* idx, int64_t n) {
    if (path.empty()) throw std::invalid_argument("Empty output file name specified!");
    std::ofstream f(path, std::ios::trunc);
    if (!f.is_open()) throw IoError("cannot create " + path);
    f << std::setprecision(std::numeric_limits<double>::digits10 + 2);
    for (int64_t i = 0; i < n; ++i) f << std::sqrt(std::fabs(d2[i])) << " " << idx[i] << "\n";
}

void write_profile_bin(const std::string& path, const double* d2, const int64_t* idx, int64_t n) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f.is_open()) throw IoError("cannot create " + path);
    write_header(f, kFmtProfile, (uint64_t)n);
    std::vector<char> buf(16 * (size_t)std::min<int64_t>(n, 1 << 16));
    for (int64_t i0 = 0; i0 < n; i0 += 1 << 16) {
        const int64_t c = std::min<int64_t>(n - i0, 1 << 16);
        for (int64_t k = 0; k < c; ++k) {
            const uint64_t u = (uint64_t)idx[i0 + k];
            std::memcpy(&buf[16 * k], &d2[i0 + k], 8);
            std::memcpy(&buf[16 * k + 8], &u, 8);
        }
        f.write(buf.data(), 16 * c);
    }
}

void read_profile_bin(const std::string& path, std::vector<double>& d2, std::vector<int64_t>& idx) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) throw IoError("Could not open profile file " + path);
    const Header h = read_header(f, kFmtProfile, path);
    check_count(f, h, 16, "profile", path);
    d2.resize(h.count);
    idx.resize(h.count);
    std::vector<char> buf(16 * (size_t)h.count);
    f.read(buf.data(), buf.size());
    if (!f) throw IoError("truncated profile file " + path);
    for (uint64_t i = 0; i < h.count; ++i) {
        uint64_t u;
        std::memcpy(&d2[i], &buf[16 * i], 8);
        std::memcpy(&u, &buf[16 * i + 8], 8);
        idx[i] = (int64_t)u;
    }
}

}  // namespace io
}  // namespace matrix_profile
