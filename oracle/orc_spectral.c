/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle (checker).  FP64 restatement of the
 * reference's spectral operators and NS step; see orc_spectral.h.  The
 * arithmetic of each operator follows the reference expression by expression
 * (std::complex semantics: (0,k)*(a,b) = (0*a - k*b, 0*b + k*a), complex /=
 * double divides both parts) so the oracle can be compared bit-for-bit with
 * the reference built against the same FFT.
 */
#include "orc_spectral.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "orc_fft.h"

#define IDX(i, j, k) ((i) + nx * ((j) + ny * (k)))

double orc_freq(int64_t i, int64_t n) {
  /* src/Scalar.cpp:201-202 */
  if (i <= n / 2) return (double)i;
  return -1. * (double)n + (double)i;
}

void orc_transform(double* f, int64_t nx, int64_t ny, int64_t nz, int dir) {
  const orc_plan* py = orc_plan_cached(ny, dir);
  const orc_plan* px = orc_plan_cached(nx, dir);
  const orc_plan* pz = orc_plan_cached(nz, dir);
  /* columns: y lines of each z plane, stride nx (src/Scalar.cpp:419-444) */
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nz; k++)
    orc_execute_many(py, f + 2 * k * nx * ny, nx, nx, 1);
  /* rows: contiguous x lines (src/Scalar.cpp:476-505, single rank) */
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nz; k++)
    orc_execute_many(px, f + 2 * k * nx * ny, 1, ny, nx);
  /* z lines, stride nx*ny (src/Scalar.cpp:533-566) */
  const int64_t lines = nx * ny;
#pragma omp parallel for schedule(static)
  for (int64_t m0 = 0; m0 < lines; m0 += 8) {
    int64_t nb = lines - m0 < 8 ? lines - m0 : 8;
    orc_execute_many(pz, f + 2 * m0, nx * ny, nb, 1);
  }
}

void orc_zero_high_modes(double* f, int64_t nx, int64_t ny, int64_t nz) {
  /* src/Scalar.cpp:336-370 */
  int64_t hx = nx / 2, hy = ny / 2, hz = nz / 2;
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++) {
      double* p = f + 2 * IDX(hx, j, k);
      p[0] = 0;
      p[1] = 0;
    }
  for (int64_t k = 0; k < nz; k++)
    for (int64_t i = 0; i < nx; i++) {
      double* p = f + 2 * IDX(i, hy, k);
      p[0] = 0;
      p[1] = 0;
    }
  for (int64_t j = 0; j < ny; j++)
    for (int64_t i = 0; i < nx; i++) {
      double* p = f + 2 * IDX(i, j, hz);
      p[0] = 0;
      p[1] = 0;
    }
}

void orc_forward(double* f, int64_t nx, int64_t ny, int64_t nz, int zero) {
  orc_transform(f, nx, ny, nz, -1);
  if (zero) orc_zero_high_modes(f, nx, ny, nz);
}

void orc_inverse(double* f, int64_t nx, int64_t ny, int64_t nz) {
  orc_transform(f, nx, ny, nz, 1);
  const int64_t n = nx * ny * nz;
  const double N = (double)(uint64_t)n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    f[2 * i] /= N;
    f[2 * i + 1] /= N;
  }
}

/* (0,k) * (a,b) as std::complex evaluates it */
static inline void ik_mul(double k, const double* z, double* re, double* im) {
  *re = 0.0 * z[0] - k * z[1];
  *im = 0.0 * z[1] + k * z[0];
}

void orc_gradient(const double* f, double* gx, double* gy, double* gz, int64_t nx,
                  int64_t ny, int64_t nz) {
  double* g[3] = {gx, gy, gz};
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++)
      for (int64_t i = 0; i < nx; i++) {
        double fr[3] = {orc_freq(i, nx), orc_freq(j, ny), orc_freq(k, nz)};
        int64_t n = IDX(i, j, k);
        for (int d = 0; d < 3; d++) ik_mul(fr[d], f + 2 * n, &g[d][2 * n], &g[d][2 * n + 1]);
      }
}

void orc_laplacian(const double* f, double* out, int64_t nx, int64_t ny, int64_t nz) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++)
      for (int64_t i = 0; i < nx; i++) {
        double a = orc_freq(i, nx), b = orc_freq(j, ny), c = orc_freq(k, nz);
        double s = -(a * a + b * b + c * c);
        int64_t n = IDX(i, j, k);
        out[2 * n] = s * f[2 * n];
        out[2 * n + 1] = s * f[2 * n + 1];
      }
}

void orc_laplacian_inverse(double* f, double a, double b, int64_t nx, int64_t ny,
                           int64_t nz) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++)
      for (int64_t i = 0; i < nx; i++) {
        double fr[3] = {orc_freq(i, nx), orc_freq(j, ny), orc_freq(k, nz)};
        double sum = 0;
        for (int d = 0; d < 3; d++) sum += fr[d] * fr[d];
        if (sum != 0) {
          double den = a - b * sum;
          int64_t n = IDX(i, j, k);
          f[2 * n] /= den;
          f[2 * n + 1] /= den;
        }
      }
}

void orc_curl(const double* const v[3], double* const out[3], int64_t nx, int64_t ny,
              int64_t nz) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++)
      for (int64_t i = 0; i < nx; i++) {
        double f[3] = {orc_freq(i, nx), orc_freq(j, ny), orc_freq(k, nz)};
        int64_t n = IDX(i, j, k);
        double ar, ai, br, bi;
        /* src/Vector.cpp:105-110 */
        ik_mul(f[1], v[2] + 2 * n, &ar, &ai);
        ik_mul(f[2], v[1] + 2 * n, &br, &bi);
        out[0][2 * n] = ar - br;
        out[0][2 * n + 1] = ai - bi;
        ik_mul(f[2], v[0] + 2 * n, &ar, &ai);
        ik_mul(f[0], v[2] + 2 * n, &br, &bi);
        out[1][2 * n] = ar - br;
        out[1][2 * n + 1] = ai - bi;
        ik_mul(f[0], v[1] + 2 * n, &ar, &ai);
        ik_mul(f[1], v[0] + 2 * n, &br, &bi);
        out[2][2 * n] = ar - br;
        out[2][2 * n + 1] = ai - bi;
      }
}

void orc_divergence(const double* const v[3], double* out, int64_t nx, int64_t ny,
                    int64_t nz) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++)
      for (int64_t i = 0; i < nx; i++) {
        double f[3] = {orc_freq(i, nx), orc_freq(j, ny), orc_freq(k, nz)};
        int64_t n = IDX(i, j, k);
        double sr = 0, si = 0; /* src/Vector.cpp:139-142 */
        for (int d = 0; d < 3; d++) {
          double tr, ti;
          ik_mul(f[d], v[d] + 2 * n, &tr, &ti);
          sr += tr;
          si += ti;
        }
        out[2 * n] = sr;
        out[2 * n + 1] = si;
      }
}

void orc_vlaplacian(const double* const v[3], double* const out[3], int64_t nx,
                    int64_t ny, int64_t nz) {
  for (int d = 0; d < 3; d++) orc_laplacian(v[d], out[d], nx, ny, nz);
}

static inline void cmul(const double* a, const double* b, double* re, double* im) {
  *re = a[0] * b[0] - a[1] * b[1];
  *im = a[0] * b[1] + a[1] * b[0];
}

void orc_cross(const double* const a[3], const double* const b[3],
               double* const out[3], int64_t nx, int64_t ny, int64_t nz, int zero) {
  const int64_t n = nx * ny * nz;
  const size_t bytes = sizeof(double) * 2 * (size_t)n;
  double* u[3];
  double* v[3];
  for (int d = 0; d < 3; d++) {
    u[d] = (double*)malloc(bytes);
    v[d] = (double*)malloc(bytes);
    memcpy(u[d], a[d], bytes);
    memcpy(v[d], b[d], bytes);
    orc_inverse(u[d], nx, ny, nz);
    orc_inverse(v[d], nx, ny, nz);
  }
  /* src/Vector.cpp:79-85 */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    double pr, pi, qr, qi;
    cmul(u[1] + 2 * i, v[2] + 2 * i, &pr, &pi);
    cmul(u[2] + 2 * i, v[1] + 2 * i, &qr, &qi);
    out[0][2 * i] = pr - qr;
    out[0][2 * i + 1] = pi - qi;
    cmul(u[2] + 2 * i, v[0] + 2 * i, &pr, &pi);
    cmul(u[0] + 2 * i, v[2] + 2 * i, &qr, &qi);
    out[1][2 * i] = pr - qr;
    out[1][2 * i + 1] = pi - qi;
    cmul(u[0] + 2 * i, v[1] + 2 * i, &pr, &pi);
    cmul(u[1] + 2 * i, v[0] + 2 * i, &qr, &qi);
    out[2][2 * i] = pr - qr;
    out[2][2 * i + 1] = pi - qi;
  }
  for (int d = 0; d < 3; d++) {
    orc_forward(out[d], nx, ny, nz, zero);
    free(u[d]);
    free(v[d]);
  }
}

double orc_average(const double* f, int64_t n) {
  /* src/Scalar.cpp:15-22: serial complex accumulation of |f_i| */
  double avg = 0;
  for (int64_t i = 0; i < n; i++) avg += hypot(f[2 * i], f[2 * i + 1]);
  return avg / (double)n;
}

void orc_add(const double* a, const double* b, double* out, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < 2 * n; i++) out[i] = a[i] + b[i];
}
void orc_sub(const double* a, const double* b, double* out, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < 2 * n; i++) out[i] = a[i] - b[i];
}
void orc_mul(const double* a, const double* b, double* out, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; i++) {
    double r, m;
    cmul(a + 2 * i, b + 2 * i, &r, &m);
    out[2 * i] = r;
    out[2 * i + 1] = m;
  }
}
void orc_scale(double alpha, const double* a, double* out, int64_t n) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < 2 * n; i++) out[i] = alpha * a[i];
}

/* ------------------------------------------------------------------ */
/* NS integrator (exec/ns.cpp)                                         */

typedef struct {
  double* c[3];
} vec3;

static vec3 vnew(int64_t n) {
  vec3 v;
  for (int d = 0; d < 3; d++) v.c[d] = (double*)calloc(2 * (size_t)n, sizeof(double));
  return v;
}
static void vfree(vec3 v) {
  for (int d = 0; d < 3; d++) free(v.c[d]);
}
static void vcopy(double* const dst[3], const double* const src[3], int64_t n) {
  for (int d = 0; d < 3; d++) memcpy(dst[d], src[d], sizeof(double) * 2 * (size_t)n);
}
static void vadd(vec3 a, vec3 b, vec3 out, int64_t n) {
  for (int d = 0; d < 3; d++) orc_add(a.c[d], b.c[d], out.c[d], n);
}
static void vsub(vec3 a, vec3 b, vec3 out, int64_t n) {
  for (int d = 0; d < 3; d++) orc_sub(a.c[d], b.c[d], out.c[d], n);
}
static void vscale(double s, vec3 a, vec3 out, int64_t n) {
  for (int d = 0; d < 3; d++) orc_scale(s, a.c[d], out.c[d], n);
}
#define CV(v) ((const double* const*)(v).c)

static vec3 asvec(double* const p[3]) {
  vec3 v = {{p[0], p[1], p[2]}};
  return v;
}

orc_ns* orc_ns_create(int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
                      int zero) {
  orc_ns* s = (orc_ns*)calloc(1, sizeof(orc_ns));
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  s->nu = nu;
  s->dt = dt;
  s->zero = zero;
  int64_t n = nx * ny * nz;
  for (int d = 0; d < 3; d++) {
    s->V0[d] = (double*)calloc(2 * (size_t)n, sizeof(double));
    s->V1[d] = (double*)calloc(2 * (size_t)n, sizeof(double));
    s->omega0[d] = (double*)calloc(2 * (size_t)n, sizeof(double));
    s->omega1[d] = (double*)calloc(2 * (size_t)n, sizeof(double));
    s->cross0[d] = (double*)calloc(2 * (size_t)n, sizeof(double));
  }
  return s;
}

void orc_ns_destroy(orc_ns* s) {
  if (!s) return;
  for (int d = 0; d < 3; d++) {
    free(s->V0[d]);
    free(s->V1[d]);
    free(s->omega0[d]);
    free(s->omega1[d]);
    free(s->cross0[d]);
  }
  free(s);
}

void orc_ns_bootstrap(orc_ns* s, const double* const V0[3],
                      const double* const omega0[3]) {
  const int64_t nx = s->nx, ny = s->ny, nz = s->nz, n = nx * ny * nz;
  const double nu = s->nu, K = s->dt;
  vcopy(s->V0, V0, n);
  vcopy(s->omega0, omega0, n);
  vec3 cr = vnew(n), lp = vnew(n), t = vnew(n), g = vnew(n), v1 = vnew(n);
  double* pi0 = (double*)calloc(2 * (size_t)n, sizeof(double));
  /* Pi0 = (V0.cross(omega0) + nu*V0.laplacian()).divergence()  (ns.cpp:133) */
  orc_cross(CV(asvec(s->V0)), CV(asvec(s->omega0)), cr.c, nx, ny, nz, s->zero);
  orc_vlaplacian(CV(asvec(s->V0)), lp.c, nx, ny, nz);
  vscale(nu, lp, lp, n);
  vadd(cr, lp, t, n);
  orc_divergence(CV(t), pi0, nx, ny, nz);
  orc_laplacian_inverse(pi0, 0, 1, nx, ny, nz); /* ns.cpp:134 */
  /* V1 = V0 + K*(V0.cross(omega0) + nu*V0.laplacian() - Pi0.gradient()) (ns.cpp:137) */
  orc_gradient(pi0, g.c[0], g.c[1], g.c[2], nx, ny, nz);
  vsub(t, g, t, n);
  vscale(K, t, t, n);
  vadd(asvec(s->V0), t, v1, n);
  vcopy(s->V1, CV(v1), n);
  /* omega1 = V1.curl() (ns.cpp:140) */
  orc_curl(CV(asvec(s->V1)), s->omega1, nx, ny, nz);
  /* cross0 = V0.cross(omega0) (ns.cpp:153) */
  vcopy(s->cross0, CV(cr), n);
  vfree(cr);
  vfree(lp);
  vfree(t);
  vfree(g);
  vfree(v1);
  free(pi0);
}

double orc_ns_step(orc_ns* s) {
  const int64_t nx = s->nx, ny = s->ny, nz = s->nz, n = nx * ny * nz;
  const double nu = s->nu, K = s->dt;
  vec3 c1 = vnew(n), F = vnew(n), lap1 = vnew(n), t = vnew(n), g = vnew(n),
       V = vnew(n), om = vnew(n);
  double* G = (double*)calloc(2 * (size_t)n, sizeof(double));
  double* dv = (double*)calloc(2 * (size_t)n, sizeof(double));
  /* cross1 = V1.cross(omega1) (ns.cpp:170) */
  orc_cross(CV(asvec(s->V1)), CV(asvec(s->omega1)), c1.c, nx, ny, nz, s->zero);
  /* F = K/2*(3.*cross1 - cross0) (ns.cpp:171) */
  vscale(3., c1, t, n);
  vsub(t, asvec(s->cross0), t, n);
  vscale(K / 2, t, F, n);
  /* lap1 = nu*K/2*V1.laplacian() (ns.cpp:174) */
  orc_vlaplacian(CV(asvec(s->V1)), lap1.c, nx, ny, nz);
  vscale(nu * K / 2, lap1, lap1, n);
  /* G = (V1 + lap1 + F).divergence(); G.laplacian_inverse() (ns.cpp:177-178) */
  vadd(asvec(s->V1), lap1, t, n);
  vadd(t, F, t, n);
  orc_divergence(CV(t), G, nx, ny, nz);
  orc_laplacian_inverse(G, 0, 1, nx, ny, nz);
  /* Vhalf = V1 + F - G.gradient() (ns.cpp:181) */
  orc_gradient(G, g.c[0], g.c[1], g.c[2], nx, ny, nz);
  vadd(asvec(s->V1), F, t, n);
  vsub(t, g, t, n);
  /* V = Vhalf + lap1; V[d].laplacian_inverse(1, -nu*K/2) (ns.cpp:184-187) */
  vadd(t, lap1, V, n);
  for (int d = 0; d < 3; d++) orc_laplacian_inverse(V.c[d], 1, -nu * K / 2, nx, ny, nz);
  /* omega = V.curl(); div = V.divergence() (ns.cpp:206-210) */
  orc_curl(CV(V), om.c, nx, ny, nz);
  orc_divergence(CV(V), dv, nx, ny, nz);
  double avg = orc_average(dv, n);
  /* histories (ns.cpp:213-217) */
  vcopy(s->V0, CV(asvec(s->V1)), n);
  vcopy(s->V1, CV(V), n);
  vcopy(s->omega0, CV(asvec(s->omega1)), n);
  vcopy(s->omega1, CV(om), n);
  vcopy(s->cross0, CV(c1), n);
  s->last_div_avg = avg;
  vfree(c1);
  vfree(F);
  vfree(lap1);
  vfree(t);
  vfree(g);
  vfree(V);
  vfree(om);
  free(G);
  free(dv);
  return avg;
}

double* orc_ns_field(orc_ns* s, int slot, int d) {
  switch (slot) {
    case 0: return s->V0[d];
    case 1: return s->V1[d];
    case 2: return s->omega0[d];
    case 3: return s->omega1[d];
    default: return s->cross0[d];
  }
}

/* ------------------------------------------------------------------ */
/* initial conditions                                                  */

void orc_ic_ns_vortices(double* omega_z, int64_t nx, int64_t ny, int64_t nz) {
  /* exec/ns.cpp:90-112 */
  const double width = M_PI / 8, mag = 50, dist = M_PI / 2;
  const double h0 = 2. * M_PI / nx, h1 = 2. * M_PI / ny;
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++) {
      double y = h1 * j;
      for (int64_t i = 0; i < nx; i++) {
        double x = h0 * i;
#define GAUSS(xc, yc) (exp(-pow(x - (xc), 2) / width) * exp(-pow(y - (yc), 2) / width))
        double v = mag * GAUSS(M_PI - dist, M_PI - dist) +
                   mag * GAUSS(M_PI + dist, M_PI - dist) +
                   mag * GAUSS(M_PI, M_PI + dist);
#undef GAUSS
        int64_t n = IDX(i, j, k);
        omega_z[2 * n] = v;
        omega_z[2 * n + 1] = 0;
      }
    }
}

void orc_ic_taylor_green(double* const u[3], int64_t nx, int64_t ny, int64_t nz) {
  for (int64_t k = 0; k < nz; k++) {
    double z = 2. * M_PI / nz * k;
    for (int64_t j = 0; j < ny; j++) {
      double y = 2. * M_PI / ny * j;
      for (int64_t i = 0; i < nx; i++) {
        double x = 2. * M_PI / nx * i;
        int64_t n = IDX(i, j, k);
        u[0][2 * n] = sin(x) * cos(y) * cos(z);
        u[1][2 * n] = -cos(x) * sin(y) * cos(z);
        u[2][2 * n] = 0;
        for (int d = 0; d < 3; d++) u[d][2 * n + 1] = 0;
      }
    }
  }
}

void orc_velocity_from_vorticity_z(const double* wz, double* const V0[3], int64_t nx,
                                   int64_t ny, int64_t nz) {
  const int64_t n = nx * ny * nz;
  double* psi = (double*)calloc(2 * (size_t)n, sizeof(double));
  double* g[3];
  for (int d = 0; d < 3; d++) g[d] = (double*)calloc(2 * (size_t)n, sizeof(double));
  /* exec/ns.cpp:116-127 */
  for (int64_t k = 0; k < nz; k++)
    for (int64_t j = 0; j < ny; j++)
      for (int64_t i = 0; i < nx; i++) {
        double k0 = orc_freq(i, nx), k1 = orc_freq(j, ny);
        if (k0 != 0 || k1 != 0) {
          double c = -1. / (k0 * k0 + k1 * k1);
          int64_t m = IDX(i, j, k);
          psi[2 * m] = c * wz[2 * m];
          psi[2 * m + 1] = c * wz[2 * m + 1];
        }
      }
  orc_gradient(psi, g[0], g[1], g[2], nx, ny, nz);
  /* V0[0] = -1.*grad[1]; V0[1] = grad[0] (ns.cpp:129-130) */
  orc_scale(-1., g[1], V0[0], n);
  memcpy(V0[1], g[0], sizeof(double) * 2 * (size_t)n);
  memset(V0[2], 0, sizeof(double) * 2 * (size_t)n);
  for (int d = 0; d < 3; d++) free(g[d]);
  free(psi);
}
