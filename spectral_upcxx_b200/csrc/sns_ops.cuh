// Spectral operators, element-wise arithmetic and reductions (host interface).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sns {

struct Dims {
  int nx, ny, nz;
  __host__ __device__ int64_t n() const { return (int64_t)nx * ny * nz; }
};

int op_gradient(const void* f, void* gx, void* gy, void* gz, Dims d, int prec, cudaStream_t s);
int op_laplacian(const void* f, void* out, Dims d, int prec, cudaStream_t s);
int op_laplacian_inverse(void* f, double a, double b, Dims d, int prec, cudaStream_t s);
int op_curl(const void* const in[3], void* const out[3], Dims d, int prec, cudaStream_t s);
int op_divergence(const void* const in[3], void* out, Dims d, int prec, cudaStream_t s);
int op_vlaplacian(const void* const in[3], void* const out[3], Dims d, int prec,
                  cudaStream_t s);
int op_zero_high_modes(void* f, Dims d, int prec, cudaStream_t s);
// c = u x w, complex point-wise (src/Vector.cpp:79-85)
int op_cross_pointwise(const void* const u[3], const void* const w[3], void* const c[3],
                       int64_t n, int prec, cudaStream_t s);
// out = alpha*x + beta*y (y may be null: out = alpha*x)
int op_axpby(double alpha, const void* x, double beta, const void* y, void* out, int64_t n,
             int prec, cudaStream_t s);
// out = a*b, complex element-wise
int op_mul(const void* a, const void* b, void* out, int64_t n, int prec, cudaStream_t s);
// precision conversion (c64 <-> c128, or a copy)
int op_convert(void* dst, int dst_prec, const void* src, int src_prec, int64_t n,
               cudaStream_t s);
// mean |f_i| accumulated in FP64 (src/Scalar.cpp:15-22); result on the host.
// `partials` must hold reduce_partials_count() doubles of device memory.
int op_average_abs(const void* f, int64_t n, int prec, double* partials, double* result,
                   cudaStream_t s);
int reduce_partials_count();

// Vector::cross on device fields (src/Vector.cpp:66-90) with six caller-given
// work fields; tw_axes optionally supplies the twiddle table of each axis.
int vector_cross(const void* const a[3], const void* const b[3], void* const out[3], Dims d,
                 int prec, void* const scratch[6], cudaStream_t s,
                 const void* const* tw_axes = nullptr);

}  // namespace sns
