/*
 * Minimal single-process stand-in for <mpi.h>, used only to compile the
 * reference's single-rank hot-path sources (ScrimpVertBlocked and the files it
 * pulls in) into the CPU oracle.  Test infrastructure: nothing in the product
 * library includes this header.
 *
 * Only the names those translation units mention are provided.  Every call is
 * a single-rank no-op; MPI_Wtime reads std::chrono::steady_clock.
 *
 * For the reference's binary file classes (biniobase.cpp, binproffile.cpp,
 * bintsfile.cpp; used by oracle/_ref/scrimppp_ref_bin only) the single-rank
 * subset of MPI-IO they call is emulated with POSIX file calls: struct and
 * 1-D subarray datatypes (one rank writes or reads the whole array, so a view
 * is its displacement plus the subarray's start), file views, individual and
 * collective reads and writes at the view's position or at an offset, and an
 * in-place all-gather that has nothing to gather.  Other shapes throw.
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H

#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <stdexcept>
#include <vector>

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Info;
typedef int MPI_File;
typedef int MPI_Op;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_DOUBLE 1
#define MPI_LONG 2
#define MPI_INT 3
#define MPI_INTEGER 3
#define MPI_UNSIGNED 4
#define MPI_UNSIGNED_LONG 5
#define MPI_CHAR 6
#define MPI_BYTE 7
#define MPI_UINT32_T 8
#define MPI_UINT64_T 9
#define MPI_DATATYPE_NULL 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_COMM_NULL (-1)
#define MPI_INFO_NULL 0
#define MPI_FILE_NULL 0
#define MPI_SUCCESS 0

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) { throw code; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Info_create(MPI_Info* i) { *i = 1; return MPI_SUCCESS; }
inline int MPI_Info_set(MPI_Info, const char*, const char*) { return MPI_SUCCESS; }
inline int MPI_Info_free(MPI_Info* i) { *i = MPI_INFO_NULL; return MPI_SUCCESS; }
inline double MPI_Wtime() {
    return std::chrono::duration<double>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

/* ---- single-rank MPI-IO ------------------------------------------------- */

#define MPI_ORDER_C 56
#define MPI_MODE_CREATE 1
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)
#define MPI_ERR_OTHER 15

namespace oracle_mpi {
/* a datatype: bytes of data per item, bytes spanned, start offset in a view */
struct Type {
    long size, extent, offset;
};
/* an open file: descriptor, view displacement (bytes), etype extent, position (etypes) */
struct File {
    int fd;
    long long disp;
    long etype;
    long long pos;
};
inline std::vector<Type>& types() {
    static std::vector<Type> t;
    return t;
}
inline std::vector<File>& files() {
    static std::vector<File> f;
    return f;
}
inline Type type_of(MPI_Datatype d) {
    switch (d) {
        case MPI_DOUBLE: case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_UINT64_T: return {8, 8, 0};
        case MPI_INT: case MPI_UNSIGNED: case MPI_UINT32_T: return {4, 4, 0};
        case MPI_CHAR: case MPI_BYTE: return {1, 1, 0};
        default: break;
    }
    if (d >= 100 && d - 100 < (int)types().size()) return types()[d - 100];
    throw std::runtime_error("oracle MPI stub: unknown datatype");
}
inline MPI_Datatype add_type(Type t) {
    types().push_back(t);
    return 100 + (int)types().size() - 1;
}
inline File& file_of(MPI_File f) {
    if (f < 1 || f > (int)files().size() || files()[f - 1].fd < 0)
        throw std::runtime_error("oracle MPI stub: file not open");
    return files()[f - 1];
}
inline int transfer(MPI_File fh, long long at, void* buf, int count, MPI_Datatype d, bool write) {
    File& f = file_of(fh);
    const Type t = type_of(d);
    if (t.size != t.extent) throw std::runtime_error("oracle MPI stub: non-contiguous transfer");
    const long long bytes = (long long)count * t.size;
    const long long off = f.disp + at * f.etype;
    const long long done = write ? pwrite(f.fd, buf, (size_t)bytes, off)
                                 : pread(f.fd, buf, (size_t)bytes, off);
    return done == bytes ? MPI_SUCCESS : MPI_ERR_OTHER;
}
}  // namespace oracle_mpi

inline int MPI_Type_create_struct(int count, const int* blocklens, const MPI_Aint* disps,
                                  const MPI_Datatype* types, MPI_Datatype* out) {
    long size = 0, extent = 0;
    for (int i = 0; i < count; ++i) {
        const oracle_mpi::Type t = oracle_mpi::type_of(types[i]);
        size += blocklens[i] * t.size;
        const long end = (long)disps[i] + blocklens[i] * t.extent;
        if (end > extent) extent = end;
    }
    *out = oracle_mpi::add_type({size, extent, 0});
    return MPI_SUCCESS;
}
inline int MPI_Type_create_subarray(int ndims, const int* sizes, const int* subsizes,
                                    const int* starts, int, MPI_Datatype old, MPI_Datatype* out) {
    if (ndims != 1) throw std::runtime_error("oracle MPI stub: only 1-D subarrays");
    const oracle_mpi::Type t = oracle_mpi::type_of(old);
    *out = oracle_mpi::add_type({subsizes[0] * t.size, sizes[0] * t.extent, starts[0] * t.extent});
    return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype* d) { *d = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
inline int MPI_Type_get_extent(MPI_Datatype d, MPI_Aint* lb, MPI_Aint* extent) {
    *lb = 0;
    *extent = oracle_mpi::type_of(d).extent;
    return MPI_SUCCESS;
}
inline int MPI_File_open(MPI_Comm, const char* path, int amode, MPI_Info, MPI_File* fh) {
    const int flags = (amode & MPI_MODE_WRONLY) ? (O_WRONLY | ((amode & MPI_MODE_CREATE) ? O_CREAT : 0))
                                                : O_RDONLY;
    const int fd = open(path, flags, 0644);
    if (fd < 0) return MPI_ERR_OTHER;
    oracle_mpi::files().push_back({fd, 0, 1, 0});
    *fh = (int)oracle_mpi::files().size();
    return MPI_SUCCESS;
}
inline int MPI_File_close(MPI_File* fh) {
    oracle_mpi::File& f = oracle_mpi::file_of(*fh);
    close(f.fd);
    f.fd = -1;
    *fh = MPI_FILE_NULL;
    return MPI_SUCCESS;
}
inline int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                             const char*, MPI_Info) {
    oracle_mpi::File& f = oracle_mpi::file_of(fh);
    f.disp = disp + oracle_mpi::type_of(filetype).offset;
    f.etype = oracle_mpi::type_of(etype).extent;
    f.pos = 0;
    return MPI_SUCCESS;
}
inline int MPI_File_set_size(MPI_File fh, MPI_Offset size) {
    return ftruncate(oracle_mpi::file_of(fh).fd, (off_t)size) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}
inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void* buf, int count, MPI_Datatype d,
                             MPI_Status*) {
    return oracle_mpi::transfer(fh, off, const_cast<void*>(buf), count, d, true);
}
inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void* buf, int count, MPI_Datatype d,
                            MPI_Status*) {
    return oracle_mpi::transfer(fh, off, buf, count, d, false);
}
inline int MPI_File_write_all(MPI_File fh, const void* buf, int count, MPI_Datatype d, MPI_Status*) {
    oracle_mpi::File& f = oracle_mpi::file_of(fh);
    const int rc = oracle_mpi::transfer(fh, f.pos, const_cast<void*>(buf), count, d, true);
    f.pos += (long long)count * oracle_mpi::type_of(d).extent / f.etype;
    return rc;
}
inline int MPI_File_read_all(MPI_File fh, void* buf, int count, MPI_Datatype d, MPI_Status*) {
    oracle_mpi::File& f = oracle_mpi::file_of(fh);
    const int rc = oracle_mpi::transfer(fh, f.pos, buf, count, d, false);
    f.pos += (long long)count * oracle_mpi::type_of(d).extent / f.etype;
    return rc;
}
inline int MPI_File_read(MPI_File fh, void* buf, int count, MPI_Datatype d, MPI_Status* s) {
    return MPI_File_read_all(fh, buf, count, d, s);
}
inline int MPI_File_get_position(MPI_File fh, MPI_Offset* off) {
    *off = oracle_mpi::file_of(fh).pos;
    return MPI_SUCCESS;
}
inline int MPI_File_get_byte_offset(MPI_File fh, MPI_Offset off, MPI_Offset* disp) {
    const oracle_mpi::File& f = oracle_mpi::file_of(fh);
    *disp = f.disp + off * f.etype;
    return MPI_SUCCESS;
}
inline int MPI_Allgatherv(const void* send, int, MPI_Datatype, void*, const int*, const int*,
                          MPI_Datatype, MPI_Comm) {
    if (send != MPI_IN_PLACE) throw std::runtime_error("oracle MPI stub: only in-place all-gather");
    return MPI_SUCCESS;  /* one rank: its slice is already in place */
}

#endif
