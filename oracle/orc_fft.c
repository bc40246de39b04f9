/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle.  FP64 mixed-radix Stockham FFT that
 * stands in for FFTW3 (called by the reference at src/FFT1D.cpp:23-52 and
 * src/FFT1D.cpp:95-101).  See orc_fft.h for the conventions.
 *
 * Stockham DIT recursion used here.  With n = p_1 ... p_m, after a stage the
 * work array holds y[k, j] (k < r = n/L sub-sequence index, j < L frequency)
 * at position k + r*j.  A radix-p stage (L' = L p, r' = r/p) computes
 *     y'[k, j + L s] = sum_q W_p^{qs} * W_n^{q j r'} * y[k + r' q, j]
 * so the innermost loop over k is unit stride.
 */
#include "orc_fft.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define ORC_MAX_FACTORS 64

struct orc_plan {
  int64_t n;
  int sign;
  int nf;
  int64_t fac[ORC_MAX_FACTORS];
  double* w; /* w[2m], w[2m+1] = cos, sin of sign*2*pi*m/n, m < n */
};

void orc_cis(int64_t m, int64_t n, double* c, double* s) {
  m %= n;
  if (m < 0) m += n;
  int64_t m8 = 8 * m;
  int64_t oct = m8 / n;
  int64_t rem = m8 - oct * n;
  double t;
  if (oct & 1)
    t = (M_PI / 4) * ((double)(n - rem) / (double)n);
  else
    t = (M_PI / 4) * ((double)rem / (double)n);
  double ct = cos(t), st = sin(t), x, y;
  switch (oct) {
    case 0: x = ct; y = st; break;
    case 1: x = st; y = ct; break;
    case 2: x = -st; y = ct; break;
    case 3: x = -ct; y = st; break;
    case 4: x = -ct; y = -st; break;
    case 5: x = -st; y = -ct; break;
    case 6: x = st; y = -ct; break;
    default: x = ct; y = -st; break;
  }
  *c = x;
  *s = y;
}

orc_plan* orc_plan_create(int64_t n, int sign) {
  if (n < 1) return NULL;
  orc_plan* p = (orc_plan*)calloc(1, sizeof(orc_plan));
  p->n = n;
  p->sign = sign < 0 ? -1 : 1;
  int64_t r = n;
  while (r % 4 == 0) { p->fac[p->nf++] = 4; r /= 4; }
  while (r % 2 == 0) { p->fac[p->nf++] = 2; r /= 2; }
  for (int64_t f = 3; r > 1;) {
    if (r % f == 0) { p->fac[p->nf++] = f; r /= f; }
    else f += 2;
  }
  p->w = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  for (int64_t m = 0; m < n; m++) {
    double c, s;
    orc_cis(m, n, &c, &s);
    p->w[2 * m] = c;
    p->w[2 * m + 1] = p->sign * s;
  }
  return p;
}

void orc_plan_destroy(orc_plan* p) {
  if (!p) return;
  free(p->w);
  free(p);
}

int64_t orc_plan_n(const orc_plan* p) { return p->n; }
int orc_plan_sign(const orc_plan* p) { return p->sign; }

/* One Stockham stage: src -> dst, radix p, L sub-transform length so far. */
static void stage(const orc_plan* P, const double* src, double* dst, int64_t p,
                  int64_t L) {
  const int64_t n = P->n;
  const int64_t r = n / L, rp = r / p;
  const double* w = P->w;
  const double sg = (double)P->sign;
  for (int64_t j = 0; j < L; j++) {
    double tw[2 * 16];
    double* twd = NULL;
    if (p <= 16) {
      twd = tw;
    } else {
      twd = (double*)malloc(sizeof(double) * 2 * (size_t)p);
    }
    for (int64_t q = 0; q < p; q++) {
      int64_t m = (q * j * rp) % n;
      twd[2 * q] = w[2 * m];
      twd[2 * q + 1] = w[2 * m + 1];
    }
    for (int64_t k = 0; k < rp; k++) {
      double in[2 * 16];
      double* a = in;
      double* big = NULL;
      if (p > 16) big = a = (double*)malloc(sizeof(double) * 2 * (size_t)p);
      for (int64_t q = 0; q < p; q++) {
        const double* x = src + 2 * (k + rp * (q + p * j));
        double xr = x[0], xi = x[1];
        double cr = twd[2 * q], ci = twd[2 * q + 1];
        if (q == 0) {
          a[0] = xr;
          a[1] = xi;
        } else {
          a[2 * q] = xr * cr - xi * ci;
          a[2 * q + 1] = xr * ci + xi * cr;
        }
      }
#define OUT(s) (dst + 2 * (k + rp * (j + L * (s))))
      if (p == 2) {
        double* o0 = OUT(0);
        double* o1 = OUT(1);
        o0[0] = a[0] + a[2];
        o0[1] = a[1] + a[3];
        o1[0] = a[0] - a[2];
        o1[1] = a[1] - a[3];
      } else if (p == 4) {
        double t0r = a[0] + a[4], t0i = a[1] + a[5];
        double t1r = a[0] - a[4], t1i = a[1] - a[5];
        double t2r = a[2] + a[6], t2i = a[3] + a[7];
        double dr = a[2] - a[6], di = a[3] - a[7];
        /* (dr + i di) * (sign i) = sign*(-di + i dr) */
        double t3r = -sg * di, t3i = sg * dr;
        double* o0 = OUT(0);
        double* o1 = OUT(1);
        double* o2 = OUT(2);
        double* o3 = OUT(3);
        o0[0] = t0r + t2r; o0[1] = t0i + t2i;
        o2[0] = t0r - t2r; o2[1] = t0i - t2i;
        o1[0] = t1r + t3r; o1[1] = t1i + t3i;
        o3[0] = t1r - t3r; o3[1] = t1i - t3i;
      } else if (p == 3) {
        const double h = 0.86602540378443864676; /* sqrt(3)/2 */
        double t1r = a[2] + a[4], t1i = a[3] + a[5];
        double t2r = a[2] - a[4], t2i = a[3] - a[5];
        double mr = a[0] - 0.5 * t1r, mi = a[1] - 0.5 * t1i;
        /* u = sign*h*i*t2 */
        double ur = -sg * h * t2i, ui = sg * h * t2r;
        double* o0 = OUT(0);
        double* o1 = OUT(1);
        double* o2 = OUT(2);
        o0[0] = a[0] + t1r; o0[1] = a[1] + t1i;
        o1[0] = mr + ur; o1[1] = mi + ui;
        o2[0] = mr - ur; o2[1] = mi - ui;
      } else {
        /* direct DFT of a prime factor: W_p^{m} = w[(m mod p) * n/p] */
        const int64_t np = n / p;
        for (int64_t s = 0; s < p; s++) {
          double sr = 0, si = 0;
          for (int64_t q = 0; q < p; q++) {
            int64_t m = ((q * s) % p) * np;
            double cr = w[2 * m], ci = w[2 * m + 1];
            sr += a[2 * q] * cr - a[2 * q + 1] * ci;
            si += a[2 * q] * ci + a[2 * q + 1] * cr;
          }
          double* o = OUT(s);
          o[0] = sr;
          o[1] = si;
        }
      }
#undef OUT
      if (big) free(big);
    }
    if (p > 16) free(twd);
  }
}

/* Transform one contiguous line in buf (length n); tmp is scratch of the same
 * size.  Result ends in buf. */
static void line_contig(const orc_plan* P, double* buf, double* tmp) {
  double* src = buf;
  double* dst = tmp;
  int64_t L = 1;
  for (int f = 0; f < P->nf; f++) {
    int64_t p = P->fac[f];
    stage(P, src, dst, p, L);
    L *= p;
    double* t = src;
    src = dst;
    dst = t;
  }
  if (src != buf) memcpy(buf, src, sizeof(double) * 2 * (size_t)P->n);
}

static __thread double* tls_buf = NULL;
static __thread size_t tls_cap = 0;

static double* scratch(size_t doubles) {
  if (doubles > tls_cap) {
    free(tls_buf);
    tls_buf = (double*)malloc(sizeof(double) * doubles);
    tls_cap = doubles;
  }
  return tls_buf;
}

void orc_execute_strided(const orc_plan* P, double* data, int64_t stride) {
  const int64_t n = P->n;
  if (stride == 1) {
    double* t = scratch(2 * (size_t)n);
    line_contig(P, data, t);
    return;
  }
  double* b = scratch(4 * (size_t)n);
  double* t = b + 2 * n;
  for (int64_t i = 0; i < n; i++) {
    b[2 * i] = data[2 * i * stride];
    b[2 * i + 1] = data[2 * i * stride + 1];
  }
  line_contig(P, b, t);
  for (int64_t i = 0; i < n; i++) {
    data[2 * i * stride] = b[2 * i];
    data[2 * i * stride + 1] = b[2 * i + 1];
  }
}

void orc_execute_many(const orc_plan* P, double* data, int64_t stride,
                      int64_t howmany, int64_t dist) {
  const int64_t n = P->n;
  if (stride == 1) {
    double* t = scratch(2 * (size_t)n);
    for (int64_t b = 0; b < howmany; b++) line_contig(P, data + 2 * b * dist, t);
    return;
  }
  /* Blocks of up to 8 adjacent lines when the lines are adjacent (dist == 1),
   * so each gathered row is one 128-byte run. */
  const int64_t B = (dist == 1) ? 8 : 1;
  double* buf = scratch((size_t)(2 * n * B + 2 * n));
  double* t = buf + 2 * n * B;
  for (int64_t b0 = 0; b0 < howmany; b0 += B) {
    int64_t nb = howmany - b0 < B ? howmany - b0 : B;
    for (int64_t i = 0; i < n; i++) {
      const double* row = data + 2 * (b0 * dist + i * stride);
      for (int64_t b = 0; b < nb; b++) {
        buf[2 * (b * n + i)] = row[2 * b * dist];
        buf[2 * (b * n + i) + 1] = row[2 * b * dist + 1];
      }
    }
    for (int64_t b = 0; b < nb; b++) line_contig(P, buf + 2 * b * n, t);
    for (int64_t i = 0; i < n; i++) {
      double* row = data + 2 * (b0 * dist + i * stride);
      for (int64_t b = 0; b < nb; b++) {
        row[2 * b * dist] = buf[2 * (b * n + i)];
        row[2 * b * dist + 1] = buf[2 * (b * n + i) + 1];
      }
    }
  }
}

/* ---- plan cache ---- */
typedef struct cache_ent {
  int64_t n;
  int sign;
  orc_plan* p;
  struct cache_ent* next;
} cache_ent;

static cache_ent* g_cache = NULL;
static pthread_mutex_t g_lock = PTHREAD_MUTEX_INITIALIZER;

const orc_plan* orc_plan_cached(int64_t n, int sign) {
  sign = sign < 0 ? -1 : 1;
  pthread_mutex_lock(&g_lock);
  for (cache_ent* e = g_cache; e; e = e->next) {
    if (e->n == n && e->sign == sign) {
      pthread_mutex_unlock(&g_lock);
      return e->p;
    }
  }
  cache_ent* e = (cache_ent*)malloc(sizeof(cache_ent));
  e->n = n;
  e->sign = sign;
  e->p = orc_plan_create(n, sign);
  e->next = g_cache;
  g_cache = e;
  pthread_mutex_unlock(&g_lock);
  return e->p;
}
