/* TEST INFRASTRUCTURE ONLY -- FFTW3 API subset over the oracle FFT; see
 * fftw3.h.  Plans are cheap: the twiddle tables are shared through
 * orc_plan_cached, so the reference's per-Scalar plan creation
 * (src/Scalar.cpp:105-108) costs no table rebuilds. */
#include "fftw3.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../orc_fft.h"

struct oracle_fftw_plan_s {
  int rank;
  int64_t n[3];
  const orc_plan* p[3];
  int64_t stride, dist;
  int howmany;
  double* in;
  double* out;
};

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in,
                             const int* inembed, int istride, int idist,
                             fftw_complex* out, const int* onembed, int ostride,
                             int odist, int sign, unsigned flags) {
  (void)inembed;
  (void)onembed;
  (void)ostride;
  (void)odist;
  (void)flags;
  if (rank != 1) return NULL;
  fftw_plan q = (fftw_plan)calloc(1, sizeof(*q));
  q->rank = 1;
  q->n[0] = n[0];
  q->p[0] = orc_plan_cached(n[0], sign);
  q->stride = istride;
  q->dist = idist;
  q->howmany = howmany;
  q->in = (double*)in;
  q->out = (double*)out;
  return q;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags) {
  return fftw_plan_many_dft(1, &n, 1, in, NULL, 1, 0, out, NULL, 1, 0, sign, flags);
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in,
                           fftw_complex* out, int sign, unsigned flags) {
  (void)flags;
  fftw_plan q = (fftw_plan)calloc(1, sizeof(*q));
  q->rank = 3;
  q->n[0] = n0;
  q->n[1] = n1;
  q->n[2] = n2;
  q->p[0] = orc_plan_cached(n0, sign);
  q->p[1] = orc_plan_cached(n1, sign);
  q->p[2] = orc_plan_cached(n2, sign);
  q->in = (double*)in;
  q->out = (double*)out;
  return q;
}

static void run(const fftw_plan q, double* in, double* out) {
  if (q->rank == 1) {
    for (int b = 0; b < q->howmany; b++) {
      double* src = in + 2 * (int64_t)b * q->dist;
      double* dst = out + 2 * (int64_t)b * q->dist;
      if (src != dst)
        for (int64_t i = 0; i < q->n[0]; i++) {
          dst[2 * i * q->stride] = src[2 * i * q->stride];
          dst[2 * i * q->stride + 1] = src[2 * i * q->stride + 1];
        }
      orc_execute_strided(q->p[0], dst, q->stride);
    }
    return;
  }
  /* row-major n0 x n1 x n2, last index fastest */
  const int64_t n0 = q->n[0], n1 = q->n[1], n2 = q->n[2];
  if (in != out) memcpy(out, in, sizeof(double) * 2 * (size_t)(n0 * n1 * n2));
  for (int64_t a = 0; a < n0 * n1; a++) orc_execute_strided(q->p[2], out + 2 * a * n2, 1);
  for (int64_t a = 0; a < n0; a++)
    for (int64_t c = 0; c < n2; c++)
      orc_execute_strided(q->p[1], out + 2 * (a * n1 * n2 + c), n2);
  for (int64_t b = 0; b < n1 * n2; b++) orc_execute_strided(q->p[0], out + 2 * b, n1 * n2);
}

void fftw_execute(const fftw_plan p) { run(p, p->in, p->out); }
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
  run(p, (double*)in, (double*)out);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }
int fftw_alignment_of(double* p) { return (int)((uintptr_t)p % 16); }
void* fftw_malloc(unsigned long n) { return malloc(n); }
void fftw_free(void* p) { free(p); }
