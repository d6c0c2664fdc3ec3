/*
 * Link-time stand-ins for the reference's MPI-IO binary file classes
 * (biniobase.h, bintsfile.hpp, binproffile.h).  The oracle build only runs the
 * reference's ASCII path and its in-memory hot path, so every binary-I/O entry
 * point here throws.  Test infrastructure only; nothing in the product links it.
 */
#include <stdexcept>
#include <string>

#include <biniobase.h>
#include <binproffile.h>
#include <bintsfile.hpp>

static void binio_unavailable() {
    throw std::runtime_error("binary MPI-IO is not part of the oracle build; use ASCII files");
}

BinIOBase::BinIOBase(const std::string& path, const MPI_Comm comm, const MPI_Info& fileinfo)
    : _path(path), _access_mode(UNDEFINED), _file_handle(MPI_FILE_NULL), _comm(comm), _rank(0),
      _header(), _fileinfo(fileinfo) {}
BinIOBase::~BinIOBase() {}

BinTsFileMPI::BinTsFileMPI(const std::string& path, const MPI_Comm comm, const MPI_Info& fileinfo)
    : BinIOBase(path, comm, fileinfo) { binio_unavailable(); }
BinTsFileMPI::~BinTsFileMPI() {}
unsigned long BinTsFileMPI::get_ts_len() { binio_unavailable(); return 0; }
int BinTsFileMPI::read_total_ts(matrix_profile::tsa_dtype* const, const size_t, const bool) {
    binio_unavailable();
    return 0;
}
unsigned int BinTsFileMPI::get_file_format_version() { return _fmt_version; }

BinProfFile::BinProfFile(const std::string& path, const MPI_Comm comm, const MPI_Info& fileinfo)
    : BinIOBase(path, comm, fileinfo) { binio_unavailable(); }
BinProfFile::~BinProfFile() {}
void BinProfFile::write_matrix_profile(const matrix_profile::tsa_dtype* const,
                                       const matrix_profile::idx_dtype* const,
                                       matrix_profile::idx_dtype) {
    binio_unavailable();
}
