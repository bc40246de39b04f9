// TEST INFRASTRUCTURE ONLY -- a project-written extern "C" entry layer over
// the reference's own classes (src/Scalar.cpp, src/Vector.cpp,
// src/Operators.cpp), compiled together with those sources in place by
// oracle/Makefile into oracle/_ref/.  Python tests call it through ctypes to
// pin the C restatement (orc_spectral.c) against the reference itself, and
// bench.py --impl reference times it on the host cores.  Fields cross this
// interface as interleaved complex doubles in the reference layout.
#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "DataObjects.H"
#include "Particle.H"

namespace {

array<INT, DIM> dims_of(int64_t nx, int64_t ny, int64_t nz) {
  return array<INT, DIM>{(INT)nx, (INT)ny, (INT)nz};
}

void load(Scalar& s, const double* src) {
  const INT n = s.localSize();
  for (INT i = 0; i < n; i++) s[i] = cdouble(src[2 * i], src[2 * i + 1]);
}

void store(const Scalar& s, double* dst) {
  const INT n = s.localSize();
  for (INT i = 0; i < n; i++) {
    cdouble v = s[i];
    dst[2 * i] = v.real();
    dst[2 * i + 1] = v.imag();
  }
}

void loadv(Vector& v, const double* const src[3]) {
  for (int d = 0; d < DIM; d++) load(v[d], src[d]);
}

void storev(const Vector& v, double* const dst[3]) {
  for (int d = 0; d < DIM; d++) store(v[d], dst[d]);
}

}  // namespace

extern "C" {

int ref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  int t = 1;
#pragma omp parallel
  {
#pragma omp single
    t = omp_get_num_threads();
  }
  return t;
}

int ref_zero_enabled(void) {
#ifdef ZERO
  return 1;
#else
  return 0;
#endif
}

// Scalar::forward (src/Scalar.cpp:208-215) on a physical field.
void ref_forward(double* f, int64_t nx, int64_t ny, int64_t nz) {
  Scalar s(dims_of(nx, ny, nz), true);
  load(s, f);
  s.forward();
  store(s, f);
}

// Scalar::inverse (src/Scalar.cpp:217-229) on a Fourier field.
void ref_inverse(double* f, int64_t nx, int64_t ny, int64_t nz) {
  Scalar s(dims_of(nx, ny, nz), false);
  load(s, f);
  s.inverse();
  store(s, f);
}

// exec/fft.cpp:52-58: `nruns` forward+inverse pairs; returns the minimum
// wall time of one pair in seconds.  f is overwritten by the last round trip.
double ref_fft_roundtrip(double* f, int64_t nx, int64_t ny, int64_t nz, int nruns) {
  Scalar s(dims_of(nx, ny, nz), true);
  load(s, f);
  double best = 1e300;
  for (int r = 0; r < nruns; r++) {
    double t0 = omp_get_wtime();
    s.forward();
    s.inverse();
    double el = omp_get_wtime() - t0;
    if (el < best) best = el;
  }
  store(s, f);
  return best;
}

void ref_gradient(const double* f, double* gx, double* gy, double* gz, int64_t nx,
                  int64_t ny, int64_t nz) {
  Scalar s(dims_of(nx, ny, nz), false);
  load(s, f);
  Vector g = s.gradient();
  double* out[3] = {gx, gy, gz};
  storev(g, out);
}

void ref_laplacian(const double* f, double* out, int64_t nx, int64_t ny, int64_t nz) {
  Scalar s(dims_of(nx, ny, nz), false);
  load(s, f);
  Scalar l = s.laplacian();
  store(l, out);
}

void ref_laplacian_inverse(double* f, double a, double b, int64_t nx, int64_t ny,
                           int64_t nz) {
  Scalar s(dims_of(nx, ny, nz), false);
  load(s, f);
  s.laplacian_inverse(a, b);
  store(s, f);
}

void ref_curl(const double* const v[3], double* const out[3], int64_t nx, int64_t ny,
              int64_t nz) {
  Vector a(dims_of(nx, ny, nz), false);
  loadv(a, v);
  Vector c = a.curl();
  storev(c, out);
}

void ref_divergence(const double* const v[3], double* out, int64_t nx, int64_t ny,
                    int64_t nz) {
  Vector a(dims_of(nx, ny, nz), false);
  loadv(a, v);
  Scalar d = a.divergence();
  store(d, out);
}

void ref_vlaplacian(const double* const v[3], double* const out[3], int64_t nx,
                    int64_t ny, int64_t nz) {
  Vector a(dims_of(nx, ny, nz), false);
  loadv(a, v);
  Vector l = a.laplacian();
  storev(l, out);
}

void ref_cross(const double* const a[3], const double* const b[3], double* const out[3],
               int64_t nx, int64_t ny, int64_t nz) {
  Vector va(dims_of(nx, ny, nz), false), vb(dims_of(nx, ny, nz), false);
  loadv(va, a);
  loadv(vb, b);
  Vector c = va.cross(vb);
  storev(c, out);
}

double ref_average(const double* f, int64_t nx, int64_t ny, int64_t nz) {
  Scalar s(dims_of(nx, ny, nz), false);
  load(s, f);
  return s.average();
}

// exec/ns.cpp:97-130: vortex-tube initial vorticity and the velocity built
// from its stream function.  Outputs are Fourier fields.
void ref_ns_vortex_ic(double* const V0_out[3], double* const omega0_out[3], int64_t nx,
                      int64_t ny, int64_t nz) {
  array<INT, DIM> dims = dims_of(nx, ny, nz);
  Vector omega0(dims);
  Vector V0(dims, false);
  array<INT, DIM> start = omega0.getPStart(), end = omega0.getPEnd();
  array<INT, DIM> ind = {0, 0, 0};
  array<double, DIM> h;
  const double width = M_PI / 8, mag = 50, dist = M_PI / 2;
  for (int i = 0; i < DIM; i++) h[i] = 2. * M_PI / dims[i];
  auto gaussian = [](double x, double y, double xc, double yc, double w) {
    return exp(-pow(x - xc, 2) / w) * exp(-pow(y - yc, 2) / w);
  };
  for (ind[2] = start[2]; ind[2] < end[2]; ind[2]++) {
    for (ind[1] = start[1]; ind[1] < end[1]; ind[1]++) {
      double y = h[1] * ind[1];
      for (ind[0] = start[0]; ind[0] < end[0]; ind[0]++) {
        double x = h[0] * ind[0];
        omega0[2][ind] = mag * gaussian(x, y, M_PI - dist, M_PI - dist, width) +
                         mag * gaussian(x, y, M_PI + dist, M_PI - dist, width) +
                         mag * gaussian(x, y, M_PI, M_PI + dist, width);
      }
    }
  }
  omega0.forward();
  Scalar psi(dims, false);
  for (ind[2] = start[2]; ind[2] < end[2]; ind[2]++)
    for (ind[1] = start[1]; ind[1] < end[1]; ind[1]++)
      for (ind[0] = start[0]; ind[0] < end[0]; ind[0]++) {
        array<double, DIM> k = psi.freq(ind);
        if (k[0] != 0 || k[1] != 0)
          psi[ind] = -1. / (k[0] * k[0] + k[1] * k[1]) * omega0[2][ind];
      }
  Vector grad = psi.gradient();
  V0[0] = -1. * grad[1];
  V0[1] = grad[0];
  storev(V0, V0_out);
  storev(omega0, omega0_out);
}

// The exec/ns.cpp time integration (bootstrap ns.cpp:132-153, loop
// ns.cpp:167-217) run on the reference classes from given Fourier V0 and
// omega0.  Writes the final V1, omega1, cross0 and every step's
// div.average() (div_avgs has nsteps entries; may be NULL).  Returns the
// wall time of the time-stepping loop in seconds.
double ref_ns_run(const double* const V0_in[3], const double* const omega0_in[3],
                  int64_t nx, int64_t ny, int64_t nz, double nu, double K, int nsteps,
                  double* const V1_out[3], double* const omega1_out[3],
                  double* const cross0_out[3], double* div_avgs) {
  array<INT, DIM> dims = dims_of(nx, ny, nz);
  Vector omega0(dims, false), omega1(dims, false), omega(dims, false);
  Vector V0(dims, false), V1(dims, false), V(dims, false), Vhalf(dims, false);
  Scalar Pi0(dims, false), Pi1(dims, false), G(dims, false), div(dims, false);
  loadv(V0, V0_in);
  loadv(omega0, omega0_in);

  Pi0 = (V0.cross(omega0) + nu * V0.laplacian()).divergence();
  Pi0.laplacian_inverse();
  V1 = V0 + K * (V0.cross(omega0) + nu * V0.laplacian() - Pi0.gradient());
  omega1 = V1.curl();
  Pi1 = (V1.cross(omega1) + nu * V1.laplacian()).divergence();
  Pi1.laplacian_inverse();
  G = K / 2 * (3 * Pi1 - Pi0);
  Vector F;
  Vector cross0 = V0.cross(omega0);
  Vector cross1;
  Vector lap1;

  double t0 = omp_get_wtime();
  for (int t = 1; t < nsteps + 1; t++) {
    cross1 = V1.cross(omega1);
    F = K / 2 * (3. * cross1 - cross0);
    lap1 = nu * K / 2 * V1.laplacian();
    G = (V1 + lap1 + F).divergence();
    G.laplacian_inverse();
    Vhalf = V1 + F - G.gradient();
    V = Vhalf + lap1;
    for (int d = 0; d < DIM; d++) V[d].laplacian_inverse(1, -nu * K / 2);
    omega = V.curl();
    div = V.divergence();
    double avg = div.average();
    if (div_avgs) div_avgs[t - 1] = avg;
    V0 = V1;
    V1 = V;
    omega0 = omega1;
    omega1 = omega;
    cross0 = cross1;
  }
  double el = omp_get_wtime() - t0;
  storev(V1, V1_out);
  storev(omega1, omega1_out);
  storev(cross0, cross0_out);
  return el;
}

// The exec/ns.cpp loop body (ns.cpp:167-217) continued from a given state
// (Fourier V1, omega1, cross0; updated in place).  Returns the wall time of
// the loop in seconds; loading and storing the fields are not timed.
double ref_ns_steps(double* const V1_io[3], double* const omega1_io[3],
                    double* const cross0_io[3], int64_t nx, int64_t ny, int64_t nz, double nu,
                    double K, int nsteps) {
  array<INT, DIM> dims = dims_of(nx, ny, nz);
  Vector V1(dims, false), omega1(dims, false), cross0(dims, false);
  Vector omega(dims, false), V0(dims, false), omega0(dims, false), V(dims, false),
      Vhalf(dims, false);
  Scalar G(dims, false), div(dims, false);
  loadv(V1, V1_io);
  loadv(omega1, omega1_io);
  loadv(cross0, cross0_io);
  Vector F, cross1, lap1;
  double t0 = omp_get_wtime();
  for (int t = 1; t < nsteps + 1; t++) {
    cross1 = V1.cross(omega1);
    F = K / 2 * (3. * cross1 - cross0);
    lap1 = nu * K / 2 * V1.laplacian();
    G = (V1 + lap1 + F).divergence();
    G.laplacian_inverse();
    Vhalf = V1 + F - G.gradient();
    V = Vhalf + lap1;
    for (int d = 0; d < DIM; d++) V[d].laplacian_inverse(1, -nu * K / 2);
    omega = V.curl();
    div = V.divergence();
    (void)div.average();
    V0 = V1;
    V1 = V;
    omega0 = omega1;
    omega1 = omega;
    cross0 = cross1;
  }
  double el = omp_get_wtime() - t0;
  storev(V1, V1_io);
  storev(omega1, omega1_io);
  storev(cross0, cross0_io);
  return el;
}

// Tracer particles of src/Particle.cpp: srand(seed), np default-constructed
// particles (random positions), nsteps moves through the physical velocity u
// (three complex fields); loc0 receives the initial positions, loc the final
// ones and energy each particle's 0.5 |v|^2 after the last move (np x 3 and np
// doubles).
void ref_particles(unsigned seed, int64_t np, const double* const u[3], int64_t nx, int64_t ny,
                   int64_t nz, double K, int nsteps, double* loc0, double* loc, double* energy) {
  Vector v(dims_of(nx, ny, nz));
  loadv(v, u);
  srand(seed);
  vector<Particle> parts(np);
  for (int64_t p = 0; p < np; p++) {
    array<double, DIM> x = parts[p].position();
    for (int d = 0; d < DIM; d++) loc0[3 * p + d] = x[d];
  }
  for (int t = 0; t < nsteps; t++)
    for (int64_t p = 0; p < np; p++) parts[p].move(v, K);
  for (int64_t p = 0; p < np; p++) {
    array<double, DIM> x = parts[p].position();
    for (int d = 0; d < DIM; d++) loc[3 * p + d] = x[d];
    energy[p] = parts[p].energy();
  }
}

}  // extern "C"
