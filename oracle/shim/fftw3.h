/* TEST INFRASTRUCTURE ONLY -- the part of the FFTW3 API that the reference
 * calls (src/FFT1D.cpp:23-52, 75-92, 100-101), implemented over the oracle's
 * own FP64 FFT (orc_fft.h) so the reference compiles unchanged without FFTW.
 * Semantics follow FFTW's documented interface: sign FFTW_FORWARD (-1) is
 * exp(-2 pi i jk/n), no normalisation, strided in-place transforms. */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H

#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct oracle_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in,
                             const int* inembed, int istride, int idist,
                             fftw_complex* out, const int* onembed, int ostride,
                             int odist, int sign, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in,
                           fftw_complex* out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_destroy_plan(fftw_plan p);
int fftw_alignment_of(double* p);
void* fftw_malloc(unsigned long n);
void fftw_free(void* p);

#ifdef __cplusplus
}
#endif

#endif
