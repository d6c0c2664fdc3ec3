/* Stand-in for the part of FFTW 3's C API that the reference's PreSCRIMP uses
 * (scrimppp/src/ScrimpppOrig.cpp:132-265): complex 1-D plans, execute,
 * destroy, aligned malloc/free.  TEST INFRASTRUCTURE: it exists so that the
 * reference's own PreSCRIMP source compiles here, where FFTW is not
 * installed, and serves as the oracle for mp_prescrimp.  The names and the
 * meaning of the arguments follow FFTW's documented interface (unnormalised
 * transforms, sign -1 forward, +1 backward); the transforms themselves are
 * written in oracle/ref_fftw_stub.cpp and round differently from FFTW's. */
#ifndef ORACLE_STUB_FFTW3_H
#define ORACLE_STUB_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct oracle_fft_plan* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
