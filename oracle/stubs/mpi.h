/*
 * Minimal single-process stand-in for <mpi.h>, used only to compile the
 * reference's single-rank hot-path sources (ScrimpVertBlocked and the files it
 * pulls in) into the CPU oracle.  Test infrastructure: nothing in the product
 * library includes this header.
 *
 * Only the names those translation units mention are provided.  Every call is
 * a single-rank no-op; MPI_Wtime reads std::chrono::steady_clock.
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H

#include <chrono>

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

#endif
