/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle (checker) for the spectral NS hot path.
 *
 * A plain-C restatement, in FP64, of the reference's Scalar / Vector /
 * Operators arithmetic and of the exec/ns.cpp time step.  Fields are
 * interleaved complex doubles (re, im) in the reference layout
 * n = i + nx*j + nx*ny*k, x fastest (src/Scalar.cpp:683).  Every function
 * names the reference lines it follows.  Parallel loops use OpenMP when the
 * file is built with -fopenmp.
 *
 * Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() may
 * call this code; the product never links it.
 */
#ifndef ORC_SPECTRAL_H
#define ORC_SPECTRAL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Unnormalised 3D DFT in place, y lines, then x lines, then z lines
 * (src/Scalar.cpp:400-646).  dir = -1 forward (exp(-i..)), +1 inverse. */
void orc_transform(double* f, int64_t nx, int64_t ny, int64_t nz, int dir);
/* Zero the planes i = nx/2, j = ny/2, k = nz/2 (src/Scalar.cpp:336-370). */
void orc_zero_high_modes(double* f, int64_t nx, int64_t ny, int64_t nz);
/* Scalar::forward: transform(-1) then zeroHighModes when zero != 0
 * (src/Scalar.cpp:208-215; ZERO is on in make.inc.in:9). */
void orc_forward(double* f, int64_t nx, int64_t ny, int64_t nz, int zero);
/* Scalar::inverse: transform(+1) then divide by N (src/Scalar.cpp:217-229). */
void orc_inverse(double* f, int64_t nx, int64_t ny, int64_t nz);

/* Scalar::freq (src/Scalar.cpp:198-206): k = i if i <= n/2 else i - n. */
double orc_freq(int64_t i, int64_t n);

/* Scalar::gradient (src/Scalar.cpp:245-276): g_d = i k_d f. */
void orc_gradient(const double* f, double* gx, double* gy, double* gz,
                  int64_t nx, int64_t ny, int64_t nz);
/* Scalar::laplacian (src/Scalar.cpp:278-306): -|k|^2 f. */
void orc_laplacian(const double* f, double* out, int64_t nx, int64_t ny, int64_t nz);
/* Scalar::laplacian_inverse (src/Scalar.cpp:308-334): f /= (a - b|k|^2)
 * wherever |k|^2 != 0. */
void orc_laplacian_inverse(double* f, double a, double b, int64_t nx, int64_t ny,
                           int64_t nz);
/* Vector::curl (src/Vector.cpp:92-122). */
void orc_curl(const double* const v[3], double* const out[3], int64_t nx, int64_t ny,
              int64_t nz);
/* Vector::divergence (src/Vector.cpp:124-153). */
void orc_divergence(const double* const v[3], double* out, int64_t nx, int64_t ny,
                    int64_t nz);
/* Vector::laplacian (src/Vector.cpp:155-181). */
void orc_vlaplacian(const double* const v[3], double* const out[3], int64_t nx,
                    int64_t ny, int64_t nz);
/* Vector::cross (src/Vector.cpp:66-90): inverse copies of both operands,
 * complex pointwise cross product, forward transform (with Nyquist zeroing
 * when zero != 0). */
void orc_cross(const double* const a[3], const double* const b[3],
               double* const out[3], int64_t nx, int64_t ny, int64_t nz, int zero);
/* Scalar::average (src/Scalar.cpp:15-22): mean |f_i|. */
double orc_average(const double* f, int64_t n);

/* Operators (src/Operators.cpp:9-99), element-wise over n complex values. */
void orc_add(const double* a, const double* b, double* out, int64_t n);
void orc_sub(const double* a, const double* b, double* out, int64_t n);
void orc_mul(const double* a, const double* b, double* out, int64_t n);
void orc_scale(double alpha, const double* a, double* out, int64_t n);

/* ---- the exec/ns.cpp time integrator ----
 * State (all Fourier, 3 components each): V1, omega1, cross0.  Work arrays
 * are allocated inside.  `zero` selects Nyquist zeroing in every forward
 * transform (ZERO build flag). */
typedef struct {
  int64_t nx, ny, nz;
  double nu, dt;
  int zero;
  double* V0[3];
  double* V1[3];
  double* omega0[3];
  double* omega1[3];
  double* cross0[3];
  double last_div_avg;
} orc_ns;

/* Allocates state arrays (zero-filled). */
orc_ns* orc_ns_create(int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
                      int zero);
void orc_ns_destroy(orc_ns* s);
/* Bootstrap from a Fourier velocity V0 and Fourier vorticity omega0
 * (exec/ns.cpp:132-153): Pi0, Forward-Euler V1, omega1 = curl V1,
 * cross0 = V0 x omega0. */
void orc_ns_bootstrap(orc_ns* s, const double* const V0[3],
                      const double* const omega0[3]);
/* One AB2 / projection / Crank-Nicolson step (exec/ns.cpp:167-217).  Returns
 * the divergence monitor div.average() of the new velocity. */
double orc_ns_step(orc_ns* s);
/* State array access for bindings: slot 0..4 = V0, V1, omega0, omega1,
 * cross0; component d = 0..2. */
double* orc_ns_field(orc_ns* s, int slot, int d);

/* Initial conditions used by the tests and benchmarks (physical space, real
 * part only, written into interleaved complex arrays). */
/* exec/ns.cpp:90-112: three Gaussian vortex tubes in omega_z, returns the
 * physical omega_z; the caller builds V0 as ns.cpp:113-130 does. */
void orc_ic_ns_vortices(double* omega_z, int64_t nx, int64_t ny, int64_t nz);
/* Taylor-Green: u = sin x cos y cos z, v = -cos x sin y cos z, w = 0. */
void orc_ic_taylor_green(double* const u[3], int64_t nx, int64_t ny, int64_t nz);
/* exec/ns.cpp:115-130: V0 = (-d_y psi, d_x psi, 0), psi = -omega_z/(kx^2+ky^2)
 * (Fourier omega_z in, Fourier V0 out). */
void orc_velocity_from_vorticity_z(const double* omega_z_hat, double* const V0[3],
                                   int64_t nx, int64_t ny, int64_t nz);

#ifdef __cplusplus
}
#endif

#endif
