/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the spectral NS hot path.
 *
 * Project-written FP64 mixed-radix FFT. It stands in for FFTW3, which the
 * reference calls through FFT1D (src/FFT1D.cpp:23-52 plan creation,
 * src/FFT1D.cpp:95-101 fftw_execute_dft) and which is not installed here
 * (the reference pins no FFTW version; make.inc.in:3 only names a path).
 * The algorithm is the textbook Stockham autosort DIT recursion
 * (Van Loan, "Computational Frameworks for the FFT", sec. 1.7), radices
 * 4, 2, 3, 5 and a direct DFT for any other prime factor, so every length
 * is supported.  Sign convention is FFTW's: sign = -1 computes
 * X[k] = sum_j x[j] exp(-2 pi i jk/n), sign = +1 the conjugate; neither
 * direction is normalised.
 *
 * Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() may
 * use this code, as the checker; the product never links it.
 */
#ifndef ORC_FFT_H
#define ORC_FFT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_plan orc_plan;

/* Plan a length-n transform with the given sign (+1 or -1). Thread safe. */
orc_plan* orc_plan_create(int64_t n, int sign);
void orc_plan_destroy(orc_plan* p);
int64_t orc_plan_n(const orc_plan* p);
int orc_plan_sign(const orc_plan* p);

/* In-place transform of one line of n complex doubles (interleaved re,im)
 * whose elements sit `stride` complex elements apart. Thread safe: it uses a
 * thread-local scratch buffer. */
void orc_execute_strided(const orc_plan* p, double* data, int64_t stride);

/* In-place transform of `howmany` lines. Line b starts at data + 2*b*dist,
 * elements `stride` apart. Lines are processed in blocks so strided lines are
 * gathered with cache-friendly access. */
void orc_execute_many(const orc_plan* p, double* data, int64_t stride,
                      int64_t howmany, int64_t dist);

/* Shared plan cache keyed by (n, sign); plans live until process exit. */
const orc_plan* orc_plan_cached(int64_t n, int sign);

/* cos/sin(2 pi m / n) with argument reduction to the first octant. */
void orc_cis(int64_t m, int64_t n, double* c, double* s);

#ifdef __cplusplus
}
#endif

#endif
