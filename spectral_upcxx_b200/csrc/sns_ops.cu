// Spectral operators (src/Scalar.cpp:245-370, src/Vector.cpp:66-181), the
// element-wise Operators (src/Operators.cpp:9-99) and the |f| average
// (src/Scalar.cpp:15-22) as grid-stride device kernels.  Each operator makes
// one pass over HBM; wavenumbers follow Scalar::freq.
#include "sns_common.cuh"
#include "sns_ops.cuh"

namespace sns {

namespace {

constexpr int kThreads = 256;

unsigned grid_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  const int64_t cap = (int64_t)sm_count() * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

struct Idx {
  int x, y, z;
};
__device__ __forceinline__ Idx decompose(uint32_t i, int nx, int ny) {
  const uint32_t r = i / (uint32_t)nx;
  Idx o;
  o.x = (int)(i - r * (uint32_t)nx);
  o.z = (int)(r / (uint32_t)ny);
  o.y = (int)(r - (uint32_t)o.z * (uint32_t)ny);
  return o;
}

template <typename T>
__global__ void k_gradient(const cx_t<T>* __restrict__ f, cx_t<T>* gx, cx_t<T>* gy,
                           cx_t<T>* gz, Dims d) {
  const uint32_t n = (uint32_t)d.n();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Idx p = decompose(i, d.nx, d.ny);
    const cx_t<T> v = f[i];
    gx[i] = ikmul((T)freq_i(p.x, d.nx), v);
    gy[i] = ikmul((T)freq_i(p.y, d.ny), v);
    gz[i] = ikmul((T)freq_i(p.z, d.nz), v);
  }
}

template <typename T>
__device__ __forceinline__ T k2_of(const Idx& p, const Dims& d) {
  const T a = (T)freq_i(p.x, d.nx), b = (T)freq_i(p.y, d.ny), c = (T)freq_i(p.z, d.nz);
  return a * a + b * b + c * c;
}

template <typename T>
__global__ void k_laplacian(const cx_t<T>* __restrict__ f, cx_t<T>* out, Dims d) {
  const uint32_t n = (uint32_t)d.n();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Idx p = decompose(i, d.nx, d.ny);
    out[i] = cscale(-k2_of<T>(p, d), f[i]);
  }
}

// f /= (a - b|k|^2) where |k|^2 != 0; the divisor is formed and applied in
// FP64 for both precisions.
template <typename T>
__global__ void k_laplacian_inverse(cx_t<T>* f, double a, double b, Dims d) {
  const uint32_t n = (uint32_t)d.n();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Idx p = decompose(i, d.nx, d.ny);
    const double k2 = k2_of<double>(p, d);
    if (k2 != 0.0) {
      const double den = a - b * k2;
      const cx_t<T> v = f[i];
      f[i] = mk((T)((double)v.x / den), (T)((double)v.y / den));
    }
  }
}

template <typename T>
__global__ void k_curl(const cx_t<T>* __restrict__ v0, const cx_t<T>* __restrict__ v1,
                       const cx_t<T>* __restrict__ v2, cx_t<T>* o0, cx_t<T>* o1, cx_t<T>* o2,
                       Dims d) {
  const uint32_t n = (uint32_t)d.n();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Idx p = decompose(i, d.nx, d.ny);
    const T kx = (T)freq_i(p.x, d.nx), ky = (T)freq_i(p.y, d.ny), kz = (T)freq_i(p.z, d.nz);
    const cx_t<T> a = v0[i], b = v1[i], c = v2[i];
    o0[i] = csub(ikmul(ky, c), ikmul(kz, b));
    o1[i] = csub(ikmul(kz, a), ikmul(kx, c));
    o2[i] = csub(ikmul(kx, b), ikmul(ky, a));
  }
}

template <typename T>
__global__ void k_divergence(const cx_t<T>* __restrict__ v0, const cx_t<T>* __restrict__ v1,
                             const cx_t<T>* __restrict__ v2, cx_t<T>* out, Dims d) {
  const uint32_t n = (uint32_t)d.n();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Idx p = decompose(i, d.nx, d.ny);
    const T kx = (T)freq_i(p.x, d.nx), ky = (T)freq_i(p.y, d.ny), kz = (T)freq_i(p.z, d.nz);
    out[i] = cadd(cadd(ikmul(kx, v0[i]), ikmul(ky, v1[i])), ikmul(kz, v2[i]));
  }
}

template <typename T>
__global__ void k_vlaplacian(const cx_t<T>* __restrict__ v0, const cx_t<T>* __restrict__ v1,
                             const cx_t<T>* __restrict__ v2, cx_t<T>* o0, cx_t<T>* o1,
                             cx_t<T>* o2, Dims d) {
  const uint32_t n = (uint32_t)d.n();
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Idx p = decompose(i, d.nx, d.ny);
    const T s = -k2_of<T>(p, d);
    o0[i] = cscale(s, v0[i]);
    o1[i] = cscale(s, v1[i]);
    o2[i] = cscale(s, v2[i]);
  }
}

template <typename T>
__global__ void k_zero_high_modes(cx_t<T>* f, Dims d) {
  // the three Nyquist planes (src/Scalar.cpp:336-370)
  const int64_t nxy = (int64_t)d.nx * d.ny, nyz = (int64_t)d.ny * d.nz,
                nxz = (int64_t)d.nx * d.nz;
  const int64_t total = nyz + nxz + nxy;
  const int hx = d.nx >> 1, hy = d.ny >> 1, hz = d.nz >> 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t idx;
    if (i < nyz) {
      const int64_t y = i % d.ny, z = i / d.ny;
      idx = hx + d.nx * (y + d.ny * z);
    } else if (i < nyz + nxz) {
      const int64_t q = i - nyz, x = q % d.nx, z = q / d.nx;
      idx = x + d.nx * (hy + d.ny * z);
    } else {
      const int64_t q = i - nyz - nxz;
      idx = q + nxy * hz;
    }
    f[idx] = mk((T)0, (T)0);
  }
}

template <typename T>
__global__ void k_cross(const cx_t<T>* __restrict__ u0, const cx_t<T>* __restrict__ u1,
                        const cx_t<T>* __restrict__ u2, const cx_t<T>* __restrict__ w0,
                        const cx_t<T>* __restrict__ w1, const cx_t<T>* __restrict__ w2,
                        cx_t<T>* c0, cx_t<T>* c1, cx_t<T>* c2, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cx_t<T> a = u0[i], b = u1[i], c = u2[i];
    const cx_t<T> p = w0[i], q = w1[i], r = w2[i];
    c0[i] = csub(cmul(b, r), cmul(c, q));
    c1[i] = csub(cmul(c, p), cmul(a, r));
    c2[i] = csub(cmul(a, q), cmul(b, p));
  }
}

template <typename T>
__global__ void k_axpby(T alpha, const cx_t<T>* __restrict__ x, T beta,
                        const cx_t<T>* __restrict__ y, cx_t<T>* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cx_t<T> a = x[i];
    if (y) {
      const cx_t<T> b = y[i];
      out[i] = mk(alpha * a.x + beta * b.x, alpha * a.y + beta * b.y);
    } else {
      out[i] = cscale(alpha, a);
    }
  }
}

template <typename T>
__global__ void k_mul(const cx_t<T>* __restrict__ a, const cx_t<T>* __restrict__ b, cx_t<T>* out,
                      int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = cmul(a[i], b[i]);
}

template <typename S, typename D>
__global__ void k_convert(const cx_t<S>* __restrict__ src, cx_t<D>* dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cx_t<S> v = src[i];
    dst[i] = mk((D)v.x, (D)v.y);
  }
}

constexpr int kReduceBlocks = 1024;

template <typename T>
__global__ void k_abs_partial(const cx_t<T>* __restrict__ f, int64_t n, double* partials) {
  __shared__ double sm[kThreads / 32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const cx_t<T> v = f[i];
    acc += hypot((double)v.x, (double)v.y);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < kThreads / 32; w++) s += sm[w];
    partials[blockIdx.x] = s;
  }
}

__global__ void k_sum_partials(double* partials, int count) {
  __shared__ double sm[kThreads];
  double acc = 0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partials[i];
  sm[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[count] = sm[0];
}

}  // namespace

int reduce_partials_count() { return kReduceBlocks + 1; }

template <typename T>
static inline const cx_t<T>* cp(const void* p) {
  return reinterpret_cast<const cx_t<T>*>(p);
}
template <typename T>
static inline cx_t<T>* mp(void* p) {
  return reinterpret_cast<cx_t<T>*>(p);
}

static bool dims_ok(Dims d) {
  if (d.nx < 1 || d.ny < 1 || d.nz < 1 || d.n() >= ((int64_t)1 << 32)) {
    set_error("field dimensions out of range");
    return false;
  }
  return true;
}

int op_gradient(const void* f, void* gx, void* gy, void* gz, Dims d, int prec, cudaStream_t s) {
  if (!dims_ok(d)) return ERR_ARG;
  if (prec == PREC_C128)
    k_gradient<double><<<grid_for(d.n()), kThreads, 0, s>>>(cp<double>(f), mp<double>(gx),
                                                             mp<double>(gy), mp<double>(gz), d);
  else
    k_gradient<float><<<grid_for(d.n()), kThreads, 0, s>>>(cp<float>(f), mp<float>(gx),
                                                            mp<float>(gy), mp<float>(gz), d);
  SNS_CHECK_LAUNCH("k_gradient");
  return OK;
}

int op_laplacian(const void* f, void* out, Dims d, int prec, cudaStream_t s) {
  if (!dims_ok(d)) return ERR_ARG;
  if (prec == PREC_C128)
    k_laplacian<double><<<grid_for(d.n()), kThreads, 0, s>>>(cp<double>(f), mp<double>(out), d);
  else
    k_laplacian<float><<<grid_for(d.n()), kThreads, 0, s>>>(cp<float>(f), mp<float>(out), d);
  SNS_CHECK_LAUNCH("k_laplacian");
  return OK;
}

int op_laplacian_inverse(void* f, double a, double b, Dims d, int prec, cudaStream_t s) {
  if (!dims_ok(d)) return ERR_ARG;
  if (prec == PREC_C128)
    k_laplacian_inverse<double><<<grid_for(d.n()), kThreads, 0, s>>>(mp<double>(f), a, b, d);
  else
    k_laplacian_inverse<float><<<grid_for(d.n()), kThreads, 0, s>>>(mp<float>(f), a, b, d);
  SNS_CHECK_LAUNCH("k_laplacian_inverse");
  return OK;
}

int op_curl(const void* const in[3], void* const out[3], Dims d, int prec, cudaStream_t s) {
  if (!dims_ok(d)) return ERR_ARG;
  if (prec == PREC_C128)
    k_curl<double><<<grid_for(d.n()), kThreads, 0, s>>>(
        cp<double>(in[0]), cp<double>(in[1]), cp<double>(in[2]), mp<double>(out[0]),
        mp<double>(out[1]), mp<double>(out[2]), d);
  else
    k_curl<float><<<grid_for(d.n()), kThreads, 0, s>>>(
        cp<float>(in[0]), cp<float>(in[1]), cp<float>(in[2]), mp<float>(out[0]),
        mp<float>(out[1]), mp<float>(out[2]), d);
  SNS_CHECK_LAUNCH("k_curl");
  return OK;
}

int op_divergence(const void* const in[3], void* out, Dims d, int prec, cudaStream_t s) {
  if (!dims_ok(d)) return ERR_ARG;
  if (prec == PREC_C128)
    k_divergence<double><<<grid_for(d.n()), kThreads, 0, s>>>(
        cp<double>(in[0]), cp<double>(in[1]), cp<double>(in[2]), mp<double>(out), d);
  else
    k_divergence<float><<<grid_for(d.n()), kThreads, 0, s>>>(
        cp<float>(in[0]), cp<float>(in[1]), cp<float>(in[2]), mp<float>(out), d);
  SNS_CHECK_LAUNCH("k_divergence");
  return OK;
}

int op_vlaplacian(const void* const in[3], void* const out[3], Dims d, int prec,
                  cudaStream_t s) {
  if (!dims_ok(d)) return ERR_ARG;
  if (prec == PREC_C128)
    k_vlaplacian<double><<<grid_for(d.n()), kThreads, 0, s>>>(
        cp<double>(in[0]), cp<double>(in[1]), cp<double>(in[2]), mp<double>(out[0]),
        mp<double>(out[1]), mp<double>(out[2]), d);
  else
    k_vlaplacian<float><<<grid_for(d.n()), kThreads, 0, s>>>(
        cp<float>(in[0]), cp<float>(in[1]), cp<float>(in[2]), mp<float>(out[0]),
        mp<float>(out[1]), mp<float>(out[2]), d);
  SNS_CHECK_LAUNCH("k_vlaplacian");
  return OK;
}

int op_zero_high_modes(void* f, Dims d, int prec, cudaStream_t s) {
  if (!dims_ok(d)) return ERR_ARG;
  const int64_t total = (int64_t)d.ny * d.nz + (int64_t)d.nx * d.nz + (int64_t)d.nx * d.ny;
  if (prec == PREC_C128)
    k_zero_high_modes<double><<<grid_for(total), kThreads, 0, s>>>(mp<double>(f), d);
  else
    k_zero_high_modes<float><<<grid_for(total), kThreads, 0, s>>>(mp<float>(f), d);
  SNS_CHECK_LAUNCH("k_zero_high_modes");
  return OK;
}

int op_cross_pointwise(const void* const u[3], const void* const w[3], void* const c[3],
                       int64_t n, int prec, cudaStream_t s) {
  if (prec == PREC_C128)
    k_cross<double><<<grid_for(n), kThreads, 0, s>>>(
        cp<double>(u[0]), cp<double>(u[1]), cp<double>(u[2]), cp<double>(w[0]),
        cp<double>(w[1]), cp<double>(w[2]), mp<double>(c[0]), mp<double>(c[1]),
        mp<double>(c[2]), n);
  else
    k_cross<float><<<grid_for(n), kThreads, 0, s>>>(
        cp<float>(u[0]), cp<float>(u[1]), cp<float>(u[2]), cp<float>(w[0]), cp<float>(w[1]),
        cp<float>(w[2]), mp<float>(c[0]), mp<float>(c[1]), mp<float>(c[2]), n);
  SNS_CHECK_LAUNCH("k_cross");
  return OK;
}

int op_axpby(double alpha, const void* x, double beta, const void* y, void* out, int64_t n,
             int prec, cudaStream_t s) {
  if (prec == PREC_C128)
    k_axpby<double><<<grid_for(n), kThreads, 0, s>>>(alpha, cp<double>(x), beta, cp<double>(y),
                                                      mp<double>(out), n);
  else
    k_axpby<float><<<grid_for(n), kThreads, 0, s>>>((float)alpha, cp<float>(x), (float)beta,
                                                     cp<float>(y), mp<float>(out), n);
  SNS_CHECK_LAUNCH("k_axpby");
  return OK;
}

int op_mul(const void* a, const void* b, void* out, int64_t n, int prec, cudaStream_t s) {
  if (prec == PREC_C128)
    k_mul<double><<<grid_for(n), kThreads, 0, s>>>(cp<double>(a), cp<double>(b),
                                                    mp<double>(out), n);
  else
    k_mul<float><<<grid_for(n), kThreads, 0, s>>>(cp<float>(a), cp<float>(b), mp<float>(out),
                                                   n);
  SNS_CHECK_LAUNCH("k_mul");
  return OK;
}

int op_convert(void* dst, int dst_prec, const void* src, int src_prec, int64_t n,
               cudaStream_t s) {
  if (dst_prec == src_prec) {
    const size_t es = dst_prec == PREC_C128 ? 16 : 8;
    return cuda_status(cudaMemcpyAsync(dst, src, es * n, cudaMemcpyDeviceToDevice, s),
                       "cudaMemcpyAsync");
  }
  if (dst_prec == PREC_C128)
    k_convert<float, double><<<grid_for(n), kThreads, 0, s>>>(cp<float>(src), mp<double>(dst), n);
  else
    k_convert<double, float><<<grid_for(n), kThreads, 0, s>>>(cp<double>(src), mp<float>(dst), n);
  SNS_CHECK_LAUNCH("k_convert");
  return OK;
}

int op_average_abs(const void* f, int64_t n, int prec, double* partials, double* result,
                   cudaStream_t s) {
  if (n < 1) {
    set_error("average of an empty field");
    return ERR_ARG;
  }
  int64_t b = (n + kThreads - 1) / kThreads;
  const int blocks = (int)(b < kReduceBlocks ? b : kReduceBlocks);
  if (prec == PREC_C128)
    k_abs_partial<double><<<blocks, kThreads, 0, s>>>(cp<double>(f), n, partials);
  else
    k_abs_partial<float><<<blocks, kThreads, 0, s>>>(cp<float>(f), n, partials);
  SNS_CHECK_LAUNCH("k_abs_partial");
  k_sum_partials<<<1, kThreads, 0, s>>>(partials, blocks);
  SNS_CHECK_LAUNCH("k_sum_partials");
  double sum = 0;
  cudaError_t e = cudaMemcpyAsync(&sum, partials + blocks, sizeof(double),
                                  cudaMemcpyDeviceToHost, s);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemcpyAsync(average)");
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_status(e, "cudaStreamSynchronize(average)");
  *result = sum / (double)n;
  return OK;
}

}  // namespace sns
