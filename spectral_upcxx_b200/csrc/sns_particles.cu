// Tracer particles on the GPU: the move of src/Particle.cpp:12-46 for a whole
// population at once, one thread per particle (exec/ns.cpp:157-203 moves its
// 10000 particles one by one in an OpenMP loop).
//
// A particle at x in [0, 2 pi]^3 takes the cell index ind_d = trunc(x_d / h_d)
// (the reference's INT is uint64_t), h_d = 2 pi / n_d, clamped to n_d - 2 (so
// the upper neighbour is always a grid point, without periodic wrap), the
// fractions rd_d = (x_d - ind_d h_d) / h_d, the trilinear interpolation of the real parts of the three velocity
// components, then x += v K and the wrap x >= 2 pi -> x - 2 pi, x <= 0 ->
// x + 2 pi.  The eight corner terms are summed in the reference's order with
// the reference's left-to-right products, in FP64 without fused multiply-adds,
// so a complex128 velocity gives the reference's positions to the last bit.
#include <math.h>

#include "../../include/spectral_b200.h"
#include "sns_common.cuh"

namespace sns {
namespace {

template <typename T>
__device__ __forceinline__ double re_at(const cx_t<T>* __restrict__ u, int64_t i, int64_t j,
                                        int64_t k, int64_t nx, int64_t nxy) {
  return (double)u[i + nx * j + nxy * k].x;
}

// u[{i,j,k}] * w0 * w1 * w2, evaluated as ((u * w0) * w1) * w2
__device__ __forceinline__ double term(double u, double w0, double w1, double w2) {
  return __dmul_rn(__dmul_rn(__dmul_rn(u, w0), w1), w2);
}

template <typename T>
__global__ void k_particles_move(double* __restrict__ loc, double* __restrict__ vel, int64_t np,
                                 const cx_t<T>* __restrict__ u0, const cx_t<T>* __restrict__ u1,
                                 const cx_t<T>* __restrict__ u2, int64_t nx, int64_t ny,
                                 int64_t nz, double K) {
  const double two_pi = 2 * M_PI;
  const int64_t nxy = nx * ny;
  const int64_t dims[3] = {nx, ny, nz};
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    double x[3], rd[3], om[3];
    int64_t ind[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      x[d] = loc[3 * p + d];
      const double h = __ddiv_rn(two_pi, (double)dims[d]);
      ind[d] = (int64_t)__ddiv_rn(x[d], h);
      if (ind[d] >= dims[d] - 1) ind[d] = dims[d] - 2;
      // a position outside [0, 2 pi] (never produced by the wrap from inside)
      // is clamped to the first cell instead of indexing out of the field
      if (ind[d] < 0) ind[d] = 0;
      rd[d] = __ddiv_rn(__dsub_rn(x[d], __dmul_rn((double)ind[d], h)), h);
      om[d] = __dsub_rn(1.0, rd[d]);
    }
    const int64_t i = ind[0], j = ind[1], k = ind[2];
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const cx_t<T>* __restrict__ u = d == 0 ? u0 : d == 1 ? u1 : u2;
      // corners in the order of src/Particle.cpp:27-34
      double s = term(re_at<T>(u, i, j, k, nx, nxy), om[0], om[1], om[2]);
      s = __dadd_rn(s, term(re_at<T>(u, i + 1, j, k, nx, nxy), rd[0], om[1], om[2]));
      s = __dadd_rn(s, term(re_at<T>(u, i + 1, j + 1, k, nx, nxy), rd[0], rd[1], om[2]));
      s = __dadd_rn(s, term(re_at<T>(u, i, j + 1, k, nx, nxy), om[0], rd[1], om[2]));
      s = __dadd_rn(s, term(re_at<T>(u, i, j, k + 1, nx, nxy), om[0], om[1], rd[2]));
      s = __dadd_rn(s, term(re_at<T>(u, i + 1, j, k + 1, nx, nxy), rd[0], om[1], rd[2]));
      s = __dadd_rn(s, term(re_at<T>(u, i + 1, j + 1, k + 1, nx, nxy), rd[0], rd[1], rd[2]));
      s = __dadd_rn(s, term(re_at<T>(u, i, j + 1, k + 1, nx, nxy), om[0], rd[1], rd[2]));
      v[d] = s;
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
      double y = __dadd_rn(x[d], __dmul_rn(v[d], K));
      if (y >= two_pi)
        y = __dsub_rn(y, two_pi);
      else if (y <= 0)
        y = __dadd_rn(two_pi, y);
      loc[3 * p + d] = y;
      if (vel) vel[3 * p + d] = v[d];
    }
  }
}

}  // namespace
}  // namespace sns

using namespace sns;

extern "C" int sns_particles_move(double* loc, double* vel, int64_t np, const void* const u[3],
                                  int64_t nx, int64_t ny, int64_t nz, int prec, double K,
                                  void* stream) {
  if (np < 0 || (np > 0 && (!loc || !u || !u[0] || !u[1] || !u[2]))) {
    set_error("sns_particles_move: null pointer or negative count");
    return ERR_ARG;
  }
  if (nx < 2 || ny < 2 || nz < 2) {
    set_error("sns_particles_move: every dimension must be at least 2");
    return ERR_ARG;
  }
  if (prec != PREC_C64 && prec != PREC_C128) {
    set_error("sns_particles_move: unknown precision");
    return ERR_ARG;
  }
  if (np == 0) return OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int threads = 256;
  const int64_t want = (np + threads - 1) / threads;
  const unsigned blocks = (unsigned)(want < 148 * 16 ? want : 148 * 16);
  if (prec == PREC_C128)
    k_particles_move<double><<<blocks, threads, 0, s>>>(
        loc, vel, np, reinterpret_cast<const double2*>(u[0]), reinterpret_cast<const double2*>(u[1]),
        reinterpret_cast<const double2*>(u[2]), nx, ny, nz, K);
  else
    k_particles_move<float><<<blocks, threads, 0, s>>>(
        loc, vel, np, reinterpret_cast<const float2*>(u[0]), reinterpret_cast<const float2*>(u[1]),
        reinterpret_cast<const float2*>(u[2]), nx, ny, nz, K);
  SNS_CHECK_LAUNCH("k_particles_move");
  return OK;
}
