// extern "C" entry points of include/spectral_b200.h: argument checking,
// the caching device pool, and the fused NS stepper object.
#include <cuda_runtime.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/spectral_b200.h"
#include "sns_common.cuh"
#include "sns_fft.cuh"
#include "sns_ns.cuh"
#include "sns_ens.cuh"
#include "sns_les.cuh"
#include "sns_ops.cuh"

namespace sns {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }

int cuda_status(cudaError_t e, const char* where) {
  if (e == cudaSuccess) return OK;
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? ERR_ALLOC : ERR_CUDA;
}

int sm_count() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  int& c = cached[dev & 63];
  if (c == 0) {
    if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || c <= 0)
      c = 148;
  }
  return c;
}

// ---- caching pool ----------------------------------------------------------
namespace {
struct Pool {
  std::mutex mu;
  std::map<void*, std::pair<int, size_t>> live;          // ptr -> (device, bytes)
  std::map<std::pair<int, size_t>, std::vector<void*>> free_;  // (device, bytes) -> blocks
};
Pool& pool() {
  static Pool* p = new Pool();  // never destroyed: blocks outlive static teardown
  return *p;
}
size_t round_bytes(size_t b) { return (b + 255) & ~(size_t)255; }

int trim_locked(Pool& p) {
  for (auto& kv : p.free_)
    for (void* q : kv.second) cudaFree(q);
  p.free_.clear();
  return OK;
}
}  // namespace

int pool_malloc(void** ptr, size_t bytes) {
  if (!ptr) {
    set_error("sns_malloc: null output pointer");
    return ERR_ARG;
  }
  *ptr = nullptr;
  if (bytes == 0) return OK;
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t b = round_bytes(bytes);
  Pool& p = pool();
  std::lock_guard<std::mutex> lock(p.mu);
  auto key = std::make_pair(dev, b);
  auto it = p.free_.find(key);
  if (it != p.free_.end() && !it->second.empty()) {
    *ptr = it->second.back();
    it->second.pop_back();
    p.live[*ptr] = key;
    return OK;
  }
  void* q = nullptr;
  cudaError_t e = cudaMalloc(&q, b);
  if (e != cudaSuccess) {
    cudaGetLastError();
    trim_locked(p);
    e = cudaMalloc(&q, b);
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error("sns_malloc(" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e));
      return ERR_ALLOC;
    }
  }
  p.live[q] = key;
  *ptr = q;
  return OK;
}

int pool_free(void* ptr) {
  if (!ptr) return OK;
  Pool& p = pool();
  std::lock_guard<std::mutex> lock(p.mu);
  auto it = p.live.find(ptr);
  if (it == p.live.end()) {
    set_error("sns_free: pointer not from sns_malloc");
    return ERR_ARG;
  }
  p.free_[it->second].push_back(ptr);
  p.live.erase(it);
  return OK;
}

static inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
static inline size_t esize(int prec) { return prec == PREC_C128 ? 16 : 8; }

bool check_prec(int prec) {
  if (prec != PREC_C64 && prec != PREC_C128) {
    set_error("precision must be SNS_C64 (0) or SNS_C128 (1)");
    return false;
  }
  return true;
}
bool check_dims(int64_t nx, int64_t ny, int64_t nz) {
  if (nx < 1 || ny < 1 || nz < 1 || nx > (1 << 20) || ny > (1 << 20) || nz > (1 << 20) ||
      nx * ny * nz >= ((int64_t)1 << 32)) {
    set_error("dimensions out of range");
    return false;
  }
  return true;
}
bool nonnull(const void* p, const char* what) {
  if (!p) {
    set_error(std::string(what) + ": null pointer");
    return false;
  }
  return true;
}

// Vector::cross on device fields (src/Vector.cpp:66-90), scratch = 6 fields.
int vector_cross(const void* const a[3], const void* const b[3], void* const out[3], Dims d,
                 int prec, void* const scratch[6], cudaStream_t s, const void* const* tw_axes) {
  const size_t bytes = esize(prec) * d.n();
  int rc;
  for (int i = 0; i < 3; i++) {
    if ((rc = cuda_status(cudaMemcpyAsync(scratch[i], a[i], bytes, cudaMemcpyDeviceToDevice, s),
                          "cross copy")))
      return rc;
    if ((rc = cuda_status(
             cudaMemcpyAsync(scratch[3 + i], b[i], bytes, cudaMemcpyDeviceToDevice, s),
             "cross copy")))
      return rc;
  }
  if ((rc = fft3d(scratch, 6, d.nx, d.ny, d.nz, +1, PASS_SCALE, prec, s, tw_axes))) return rc;
  const void* u[3] = {scratch[0], scratch[1], scratch[2]};
  const void* w[3] = {scratch[3], scratch[4], scratch[5]};
  if ((rc = op_cross_pointwise(u, w, out, d.n(), prec, s))) return rc;
  return fft3d(out, 3, d.nx, d.ny, d.nz, -1, PASS_ZERO_NYQUIST, prec, s, tw_axes);
}

// Half spectrum (kx = 0 .. nx/2-1) of full Fourier fields of a real field, and
// the full spectrum back by Hermitian symmetry V(-k) = conj V(k) (the kx = nx/2
// plane is zero).  Three fields (blockIdx.y).
template <typename T>
__global__ void k_half_from_full(FieldPtrs f, int nxp, int ny, int nz) {
  using C = cx_t<T>;
  const int M = nxp / 2;
  const int64_t n = (int64_t)M * ny * nz;
  const C* __restrict__ in = reinterpret_cast<const C*>(f.in[blockIdx.y]);
  C* __restrict__ out = reinterpret_cast<C*>(f.out[blockIdx.y]);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = i % M, r = i / M;
    out[i] = in[r * nxp + x];
  }
}

template <typename T>
__global__ void k_full_from_half(FieldPtrs f, int nxp, int ny, int nz) {
  using C = cx_t<T>;
  const int M = nxp / 2;
  const int64_t n = (int64_t)nxp * ny * nz;
  const C* __restrict__ in = reinterpret_cast<const C*>(f.in[blockIdx.y]);
  C* __restrict__ out = reinterpret_cast<C*>(f.out[blockIdx.y]);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % nxp);
    const int64_t r = i / nxp;
    const int y = (int)(r % ny), z = (int)(r / ny);
    C v = mk((T)0, (T)0);
    if (x < M) {
      v = in[r * M + x];
    } else if (x > M) {
      const int yy = y == 0 ? 0 : ny - y, zz = z == 0 ? 0 : nz - z;
      const C c = in[((int64_t)zz * ny + yy) * M + (nxp - x)];
      v = mk(c.x, -c.y);
    }
    out[i] = v;
  }
}

// dir = +1: full -> half; -1: half -> full.  Three fields.
int convert_half(void* const* out, const void* const* in, int nxp, int ny, int nz, int prec,
                 int dir, cudaStream_t s) {
  FieldPtrs f{};
  for (int d = 0; d < 3; d++) {
    f.in[d] = const_cast<void*>(in[d]);
    f.out[d] = out[d];
  }
  const int64_t n = dir > 0 ? (int64_t)(nxp / 2) * ny * nz : (int64_t)nxp * ny * nz;
  const dim3 grid((unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16), 3);
  if (dir > 0) {
    if (prec == PREC_C128)
      k_half_from_full<double><<<grid, 256, 0, s>>>(f, nxp, ny, nz);
    else
      k_half_from_full<float><<<grid, 256, 0, s>>>(f, nxp, ny, nz);
  } else {
    if (prec == PREC_C128)
      k_full_from_half<double><<<grid, 256, 0, s>>>(f, nxp, ny, nz);
    else
      k_full_from_half<float><<<grid, 256, 0, s>>>(f, nxp, ny, nz);
  }
  return cuda_status(cudaGetLastError(), "half-spectrum conversion");
}

// The bootstrap of ns.cpp:132-153 into V (-> V1) and C0 (-> cross0), with six
// work fields U.
int ns_bootstrap_fields(Dims d, int prec, double nu, double dt, const void* const V0[3],
                        const void* const omega0[3], void* const V[3], void* const C0[3],
                        void* const U[6], cudaStream_t s) {
  const int64_t n = d.n();
  int rc;
  // cross0 = V0 x omega0 (ns.cpp:133, 137, 153)
  if ((rc = vector_cross(V0, omega0, C0, d, prec, U, s))) return rc;
  // t = cross0 + nu * laplacian(V0), held in V
  if ((rc = op_vlaplacian(V0, V, d, prec, s))) return rc;
  for (int i = 0; i < 3; i++) {
    if ((rc = op_axpby(nu, V[i], 0.0, nullptr, V[i], n, prec, s))) return rc;
    if ((rc = op_axpby(1.0, C0[i], 1.0, V[i], V[i], n, prec, s))) return rc;
  }
  // Pi0 = ilap(div t) (ns.cpp:133-134) in U[0]; grad Pi0 in U[1..3]
  const void* t[3] = {V[0], V[1], V[2]};
  if ((rc = op_divergence(t, U[0], d, prec, s))) return rc;
  if ((rc = op_laplacian_inverse(U[0], 0.0, 1.0, d, prec, s))) return rc;
  if ((rc = op_gradient(U[0], U[1], U[2], U[3], d, prec, s))) return rc;
  // V1 = V0 + K (t - grad Pi0)  (ns.cpp:137)
  for (int i = 0; i < 3; i++) {
    if ((rc = op_axpby(1.0, V[i], -1.0, U[1 + i], V[i], n, prec, s))) return rc;
    if ((rc = op_axpby(1.0, V0[i], dt, V[i], V[i], n, prec, s))) return rc;
  }
  return OK;
}

bool vec_ok(const void* const v[3], const char* what) {
  if (!v) {
    set_error(std::string(what) + ": null vector");
    return false;
  }
  for (int d = 0; d < 3; d++)
    if (!nonnull(v[d], what)) return false;
  return true;
}

}  // namespace sns

using namespace sns;

// ---- stepper object ----------------------------------------------------------
struct sns_ns {
  NSPlan pl;
  double nu, dt;
  cudaStream_t s;
  void* V[3];
  void* C0[3];
  void* U[6];
  void* W[kNSLineWork] = {};  // z-inverted V and i kz V (K1 as a line pass)
  double* stats_part;
  double* stats_out;
  int* sync_words;  // dataflow xy pass: ticket, per-plane counters, error word
  bool stepped;
  // U holds K1's output for the current V (left there by a carrying K5); any
  // call that writes V or U other than a plain step clears it
  bool carried = false;
  // eddy-viscosity closure (none by default) and its six extra work fields
  Closure cl;
  void* U2[6] = {};
  // per-pass profiling
  bool profiling = false;
  int recorded = 0;
  std::vector<cudaEvent_t> events;  // (kNSPasses + 1) per recorded step
  // one step captured as a CUDA graph (on a private stream, after one eager
  // step has set up twiddles and kernel attributes), replayed on s
  bool use_graph = true;
  bool eager_done = false;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

void drop_graph(sns_ns* h) {
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->exec = nullptr;
  h->graph = nullptr;
}

// One step (plain or closure) queued on `s`.
int step_on(sns_ns* h, cudaStream_t s, cudaEvent_t* ev) {
  if (h->cl.model != CLOSURE_NONE) {
    void* U[kLESWork];
    for (int i = 0; i < 6; i++) {
      U[i] = h->U[i];
      U[6 + i] = h->U2[i];
    }
    h->carried = false;  // the closure step uses U as work space
    return les_step_once(h->pl, h->V, h->C0, U, h->stats_part, h->nu, h->dt, h->cl, s);
  }
  return ns_step_once(h->pl, h->V, h->C0, h->U, h->stats_part, h->sync_words, h->nu, h->dt, s,
                      ev, h->W, &h->carried);
}

int capture_step(sns_ns* h) {
  int rc = OK;
  if (!h->cap)
    rc = cuda_status(cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking),
                     "sns_ns_step(capture stream)");
  if (rc) return rc;
  if ((rc = cuda_status(cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal),
                        "sns_ns_step(capture)")))
    return rc;
  const int src = step_on(h, h->cap, nullptr);
  cudaGraph_t g = nullptr;
  rc = cuda_status(cudaStreamEndCapture(h->cap, &g), "sns_ns_step(capture)");
  if (src || rc) {
    if (g) cudaGraphDestroy(g);
    return src ? src : rc;
  }
  if ((rc = cuda_status(cudaGraphInstantiate(&h->exec, g, 0), "sns_ns_step(instantiate)"))) {
    cudaGraphDestroy(g);
    h->exec = nullptr;
    return rc;
  }
  h->graph = g;
  return OK;
}

}  // namespace

extern "C" {

const char* sns_last_error(void) { return sns::last_error(); }
int sns_version(void) { return 1; }

int sns_malloc(void** ptr, size_t bytes) { return pool_malloc(ptr, bytes); }
int sns_free(void* ptr) { return pool_free(ptr); }
int sns_pool_trim(void) {
  Pool& p = pool();
  std::lock_guard<std::mutex> lock(p.mu);
  return trim_locked(p);
}

int sns_memcpy_h2d(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return OK;
  if (!nonnull(dst, "sns_memcpy_h2d") || !nonnull(src, "sns_memcpy_h2d")) return ERR_ARG;
  return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S(stream)),
                     "sns_memcpy_h2d");
}
int sns_memcpy_d2h(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return OK;
  if (!nonnull(dst, "sns_memcpy_d2h") || !nonnull(src, "sns_memcpy_d2h")) return ERR_ARG;
  return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S(stream)),
                     "sns_memcpy_d2h");
}
int sns_memcpy_d2d(void* dst, const void* src, size_t bytes, void* stream) {
  if (bytes == 0) return OK;
  if (!nonnull(dst, "sns_memcpy_d2d") || !nonnull(src, "sns_memcpy_d2d")) return ERR_ARG;
  return cuda_status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, S(stream)),
                     "sns_memcpy_d2d");
}
int sns_memset(void* ptr, int value, size_t bytes, void* stream) {
  if (bytes == 0) return OK;
  if (!nonnull(ptr, "sns_memset")) return ERR_ARG;
  return cuda_status(cudaMemsetAsync(ptr, value, bytes, S(stream)), "sns_memset");
}
int sns_stream_synchronize(void* stream) {
  return cuda_status(cudaStreamSynchronize(S(stream)), "sns_stream_synchronize");
}
int sns_convert(void* dst, int dst_prec, const void* src, int src_prec, int64_t n,
                void* stream) {
  if (!check_prec(dst_prec) || !check_prec(src_prec)) return ERR_ARG;
  if (n < 0) {
    set_error("sns_convert: negative count");
    return ERR_ARG;
  }
  if (n == 0) return OK;
  if (!nonnull(dst, "sns_convert") || !nonnull(src, "sns_convert")) return ERR_ARG;
  return op_convert(dst, dst_prec, src, src_prec, n, S(stream));
}

int sns_fft3d_many(void* const* fields, int nfields, int64_t nx, int64_t ny, int64_t nz,
                   int dir, int flags, int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz)) return ERR_ARG;
  if (dir != 1 && dir != -1) {
    set_error("sns_fft3d: dir must be -1 (forward) or +1 (inverse)");
    return ERR_ARG;
  }
  if (flags & ~(SNS_FFT_NORMALISE | SNS_FFT_ZERO_NYQUIST)) {
    set_error("sns_fft3d: unknown flags");
    return ERR_ARG;
  }
  if (!fields || nfields < 1 || nfields > kMaxFields) {
    set_error("sns_fft3d_many: 1..12 fields");
    return ERR_ARG;
  }
  for (int i = 0; i < nfields; i++)
    if (!nonnull(fields[i], "sns_fft3d")) return ERR_ARG;
  int fl = 0;
  if (flags & SNS_FFT_NORMALISE) fl |= PASS_SCALE;
  if (flags & SNS_FFT_ZERO_NYQUIST) fl |= PASS_ZERO_NYQUIST;
  return fft3d(fields, nfields, (int)nx, (int)ny, (int)nz, dir, fl, prec, S(stream));
}

int sns_fft3d(void* field, int64_t nx, int64_t ny, int64_t nz, int dir, int flags, int prec,
              void* stream) {
  void* f[1] = {field};
  return sns_fft3d_many(f, 1, nx, ny, nz, dir, flags, prec, stream);
}

int sns_fft3d_axes(void* field, int64_t nx, int64_t ny, int64_t nz, int axes, int dir,
                   double scale, int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !nonnull(field, "sns_fft3d_axes"))
    return ERR_ARG;
  if ((dir != 1 && dir != -1) || axes < 0 || axes > 7) {
    set_error("sns_fft3d_axes: dir must be -1 or +1 and axes a mask of bits 0 (x), 1 (y), 2 (z)");
    return ERR_ARG;
  }
  if (!line_supported(nx) || !line_supported(ny) || !line_supported(nz)) {
    set_error("sns_fft3d_axes: dimensions must be powers of two up to 4096");
    return ERR_UNSUPPORTED;
  }
  const int dims[3] = {(int)nx, (int)ny, (int)nz};
  int todo[3], na = 0;
  for (int a = 0; a < 3; a++)
    if (((axes >> a) & 1) && dims[a] > 1) todo[na++] = a;
  FieldPtrs f{};
  f.n = 1;
  f.in[0] = f.out[0] = field;
  for (int i = 0; i < na; i++) {
    const int fl = (i == na - 1 && scale != 1.0) ? PASS_SCALE : 0;
    int rc = run_line_pass(axis_geo(todo[i], dims[0], dims[1], dims[2], prec), f, dir, fl, scale,
                           prec, S(stream));
    if (rc) return rc;
  }
  if (na == 0 && scale != 1.0)
    return sns_axpby(scale, field, 0.0, nullptr, field, (int64_t)nx * ny * nz, prec, stream);
  return OK;
}

int sns_forward(void* field, int64_t nx, int64_t ny, int64_t nz, int prec, void* stream) {
  return sns_fft3d(field, nx, ny, nz, -1, SNS_FFT_ZERO_NYQUIST, prec, stream);
}
int sns_inverse(void* field, int64_t nx, int64_t ny, int64_t nz, int prec, void* stream) {
  return sns_fft3d(field, nx, ny, nz, +1, SNS_FFT_NORMALISE, prec, stream);
}

namespace {
// howmany lines of n elements `stride` apart, `dist` between line starts,
// transformed in place and multiplied by `scale` when it is not 1
int fft1d_lines(void* data, int64_t n, int64_t stride, int64_t howmany, int64_t dist, int dir,
                double scale, int prec, cudaStream_t s) {
  if (!check_prec(prec)) return ERR_ARG;
  if (!nonnull(data, "sns_fft1d_many")) return ERR_ARG;
  if (n < 1 || stride < 1 || howmany < 0 || dist < 0 || (dir != 1 && dir != -1)) {
    set_error("sns_fft1d_many: bad arguments");
    return ERR_ARG;
  }
  if (n == 1 && scale != 1.0 && howmany > 0) {
    set_error("sns_fft1d_many_scaled: a scale needs lines of at least two elements");
    return ERR_UNSUPPORTED;
  }
  if (howmany == 0 || n == 1) return OK;
  if (!line_supported(n)) {
    set_error("sns_fft1d_many: n must be a power of two up to 4096");
    return ERR_UNSUPPORTED;
  }
  LineGeo g{};
  g.L = (int)n;
  g.ps = stride;
  g.nx = g.ny = g.nz = 1;
  g.axis = -1;
  const int TPL = (int)(n >= 16 ? n / 16 : 1);
  auto pow2_divisor = [](int64_t v, int cap) {
    int d = 1;
    while (d * 2 <= cap && v % (d * 2) == 0) d *= 2;
    return d;
  };
  if (dist == 1 && stride > 1) {
    g.W = pow2_divisor(howmany, std::min(prec == PREC_C128 ? 8 : 16, std::max(1, max_threads(prec) / TPL)));
    g.G = 1;
    g.gs = 0;
    g.TA = howmany / g.W;
    g.sa = g.W;
  } else {
    g.W = 1;
    g.G = pow2_divisor(howmany, std::max(1, 256 / TPL));
    g.gs = dist;
    g.TA = howmany / g.G;
    g.sa = dist * g.G;
  }
  g.TB = 1;
  g.sb = 0;
  FieldPtrs f{};
  f.n = 1;
  f.in[0] = f.out[0] = data;
  return run_line_pass(g, f, dir, scale != 1.0 ? PASS_SCALE : 0, scale, prec, s);
}
}  // namespace

int sns_fft3d_tune(int64_t nx, int64_t ny, int64_t nz, int nfields, int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz)) return ERR_ARG;
  return fft3d_tune((int)nx, (int)ny, (int)nz, nfields, prec, S(stream));
}

int sns_fft3d_check(void* stream) { return fft_tma_check(S(stream)); }

int sns_fft1d_many(void* data, int64_t n, int64_t stride, int64_t howmany, int64_t dist,
                   int dir, int prec, void* stream) {
  return fft1d_lines(data, n, stride, howmany, dist, dir, 1.0, prec, S(stream));
}

int sns_fft1d_many_scaled(void* data, int64_t n, int64_t stride, int64_t howmany, int64_t dist,
                          int dir, double scale, int prec, void* stream) {
  return fft1d_lines(data, n, stride, howmany, dist, dir, scale, prec, S(stream));
}

#define SNS_DIMS_ARGS(nx, ny, nz) Dims{(int)(nx), (int)(ny), (int)(nz)}

int sns_zero_high_modes(void* field, int64_t nx, int64_t ny, int64_t nz, int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !nonnull(field, "sns_zero_high_modes"))
    return ERR_ARG;
  return op_zero_high_modes(field, SNS_DIMS_ARGS(nx, ny, nz), prec, S(stream));
}

int sns_gradient(const void* f, void* gx, void* gy, void* gz, int64_t nx, int64_t ny, int64_t nz,
                 int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz)) return ERR_ARG;
  if (!nonnull(f, "sns_gradient") || !nonnull(gx, "sns_gradient") ||
      !nonnull(gy, "sns_gradient") || !nonnull(gz, "sns_gradient"))
    return ERR_ARG;
  return op_gradient(f, gx, gy, gz, SNS_DIMS_ARGS(nx, ny, nz), prec, S(stream));
}

int sns_laplacian(const void* f, void* out, int64_t nx, int64_t ny, int64_t nz, int prec,
                  void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz)) return ERR_ARG;
  if (!nonnull(f, "sns_laplacian") || !nonnull(out, "sns_laplacian")) return ERR_ARG;
  return op_laplacian(f, out, SNS_DIMS_ARGS(nx, ny, nz), prec, S(stream));
}

int sns_laplacian_inverse(void* f, double a, double b, int64_t nx, int64_t ny, int64_t nz,
                          int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !nonnull(f, "sns_laplacian_inverse"))
    return ERR_ARG;
  return op_laplacian_inverse(f, a, b, SNS_DIMS_ARGS(nx, ny, nz), prec, S(stream));
}


int sns_curl(const void* const v[3], void* const out[3], int64_t nx, int64_t ny, int64_t nz,
             int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !vec_ok(v, "sns_curl") ||
      !vec_ok((const void* const*)out, "sns_curl"))
    return ERR_ARG;
  return op_curl(v, out, SNS_DIMS_ARGS(nx, ny, nz), prec, S(stream));
}

int sns_divergence(const void* const v[3], void* out, int64_t nx, int64_t ny, int64_t nz,
                   int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !vec_ok(v, "sns_divergence") ||
      !nonnull(out, "sns_divergence"))
    return ERR_ARG;
  return op_divergence(v, out, SNS_DIMS_ARGS(nx, ny, nz), prec, S(stream));
}

int sns_vector_laplacian(const void* const v[3], void* const out[3], int64_t nx, int64_t ny,
                         int64_t nz, int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !vec_ok(v, "sns_vector_laplacian") ||
      !vec_ok((const void* const*)out, "sns_vector_laplacian"))
    return ERR_ARG;
  return op_vlaplacian(v, out, SNS_DIMS_ARGS(nx, ny, nz), prec, S(stream));
}

int sns_cross(const void* const a[3], const void* const b[3], void* const out[3], int64_t nx,
              int64_t ny, int64_t nz, int prec, void* stream) {
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !vec_ok(a, "sns_cross") ||
      !vec_ok(b, "sns_cross") || !vec_ok((const void* const*)out, "sns_cross"))
    return ERR_ARG;
  if (!line_supported(nx) || !line_supported(ny) || !line_supported(nz)) {
    set_error("sns_cross: dimensions must be powers of two up to 4096");
    return ERR_UNSUPPORTED;
  }
  const Dims d = SNS_DIMS_ARGS(nx, ny, nz);
  void* scratch[6] = {nullptr};
  int rc = OK;
  for (int i = 0; i < 6 && rc == OK; i++) rc = pool_malloc(&scratch[i], esize(prec) * d.n());
  if (rc == OK) rc = vector_cross(a, b, out, d, prec, scratch, S(stream));
  for (int i = 0; i < 6; i++) pool_free(scratch[i]);
  return rc;
}

int sns_average_abs(const void* f, int64_t n, int prec, double* out, void* stream) {
  if (!check_prec(prec) || !nonnull(f, "sns_average_abs") || !nonnull(out, "sns_average_abs"))
    return ERR_ARG;
  void* part = nullptr;
  int rc = pool_malloc(&part, sizeof(double) * reduce_partials_count());
  if (rc) return rc;
  rc = op_average_abs(f, n, prec, (double*)part, out, S(stream));
  pool_free(part);
  return rc;
}

int sns_axpby(double alpha, const void* x, double beta, const void* y, void* out, int64_t n,
              int prec, void* stream) {
  if (!check_prec(prec) || !nonnull(x, "sns_axpby") || !nonnull(out, "sns_axpby")) return ERR_ARG;
  if (n < 0) {
    set_error("sns_axpby: negative count");
    return ERR_ARG;
  }
  if (n == 0) return OK;
  return op_axpby(alpha, x, beta, y, out, n, prec, S(stream));
}

int sns_mul(const void* a, const void* b, void* out, int64_t n, int prec, void* stream) {
  if (!check_prec(prec) || !nonnull(a, "sns_mul") || !nonnull(b, "sns_mul") ||
      !nonnull(out, "sns_mul"))
    return ERR_ARG;
  if (n < 0) {
    set_error("sns_mul: negative count");
    return ERR_ARG;
  }
  if (n == 0) return OK;
  return op_mul(a, b, out, n, prec, S(stream));
}

// ---- fused stepper -------------------------------------------------------------
int sns_ns_create(sns_ns** handle, int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
                  int prec, void* stream) {
  return sns::ns_create(handle, nx, ny, nz, nu, dt, prec, stream, false);
}

int sns_ns_create_real(sns_ns** handle, int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
                       int prec, void* stream) {
  return sns::ns_create(handle, nx, ny, nz, nu, dt, prec, stream, true);
}

}  // extern "C"

// A stepper of complex fields, or (real) of the half spectrum of real fields.
int sns::ns_create(sns_ns** handle, int64_t nx, int64_t ny, int64_t nz, double nu, double dt,
                   int prec, void* stream, bool real) {
  if (!nonnull(handle, "sns_ns_create")) return ERR_ARG;
  *handle = nullptr;
  if (!check_prec(prec) || !check_dims(nx, ny, nz)) return ERR_ARG;
  sns_ns* h = new sns_ns();
  int rc = ns_plan(h->pl, (int)nx, (int)ny, (int)nz, prec, 0, 0, real);
  if (rc) {
    delete h;
    return rc;
  }
  h->nu = nu;
  h->dt = dt;
  h->s = S(stream);
  const size_t bytes = esize(prec) * (size_t)h->pl.nx * ny * nz;  // stored (half) rows
  void** all[12];
  for (int d = 0; d < 3; d++) {
    all[d] = &h->V[d];
    all[3 + d] = &h->C0[d];
  }
  for (int i = 0; i < 6; i++) all[6 + i] = &h->U[i];
  for (int i = 0; i < 12 && rc == OK; i++) rc = pool_malloc(all[i], bytes);
  // SNS_K1_LINES=1: K1 as a line pass of V and i kz V into five more work
  // fields, the curl formed in K2 (and a candidate of the tuner).  Measured on
  // B200 at 256^3 complex64 it loses: the z line pass runs at 3.1 TB/s like
  // the fused K1 tile (0.351 vs 0.394 ms) while the omega prologue's extra
  // loads slow K2 from 0.297 to 0.522 ms.
  const char* kl = getenv("SNS_K1_LINES");
  if (rc == OK && kl && kl[0] == '1') {
    for (int i = 0; i < kNSLineWork && rc == OK; i++) rc = pool_malloc(&h->W[i], bytes);
    if (rc == OK) h->pl.k1_lines = true;
  }
  if (rc == OK)
    rc = pool_malloc((void**)&h->stats_part,
                     sizeof(double) * 4 * std::max(h->pl.update_blocks, h->pl.sgs_blocks));
  if (rc == OK) rc = pool_malloc((void**)&h->stats_out, sizeof(double) * 4);
  if (rc == OK) rc = pool_malloc((void**)&h->sync_words, sizeof(int) * xy_sync_words((int)nz));
  if (rc == OK)
    rc = cuda_status(cudaMemsetAsync(h->sync_words, 0, sizeof(int) * xy_sync_words((int)nz), h->s),
                     "sns_ns_create");
  if (rc == OK) {
    for (int i = 0; i < 6 && rc == OK; i++)
      rc = cuda_status(cudaMemsetAsync(*all[i], 0, bytes, h->s), "sns_ns_create");
  }
  if (rc) {
    sns_ns_destroy(h);
    return rc;
  }
  h->stepped = false;
  h->carried = false;
  // SNS_GRAPH=0 launches every step's kernels directly
  if (const char* e = getenv("SNS_GRAPH")) h->use_graph = e[0] != '0';
  // SNS_TUNE=1: every new stepper tunes its plan (cached per device and shape)
  if (tune_on_first_use() && (rc = sns_ns_tune(h))) {
    sns_ns_destroy(h);
    return rc;
  }
  *handle = h;
  return OK;
}

extern "C" {

int sns_ns_destroy(sns_ns* h) {
  if (!h) return OK;
  cudaStreamSynchronize(h->s);
  for (int d = 0; d < 3; d++) {
    pool_free(h->V[d]);
    pool_free(h->C0[d]);
  }
  for (int i = 0; i < 6; i++) pool_free(h->U[i]);
  for (int i = 0; i < kNSLineWork; i++) pool_free(h->W[i]);
  pool_free(h->stats_part);
  pool_free(h->stats_out);
  pool_free(h->sync_words);
  for (int i = 0; i < 6; i++) pool_free(h->U2[i]);
  for (cudaEvent_t e : h->events) cudaEventDestroy(e);
  drop_graph(h);
  h->carried = false;
  if (h->cap) cudaStreamDestroy(h->cap);
  delete h;
  return OK;
}

int sns_ns_set_state(sns_ns* h, const void* const V1[3], const void* const cross0[3]) {
  if (!nonnull(h, "sns_ns_set_state") || !vec_ok(V1, "sns_ns_set_state") ||
      !vec_ok(cross0, "sns_ns_set_state"))
    return ERR_ARG;
  if (h->pl.real) {
    int rc = convert_half(h->V, V1, h->pl.nx_phys, h->pl.ny, h->pl.nz, h->pl.prec, +1, h->s);
    if (!rc) rc = convert_half(h->C0, cross0, h->pl.nx_phys, h->pl.ny, h->pl.nz, h->pl.prec, +1,
                               h->s);
    if (rc) return rc;
    h->stepped = false;
    h->carried = false;
    return OK;
  }
  const size_t bytes = esize(h->pl.prec) * (size_t)h->pl.nx * h->pl.ny * h->pl.nz;
  int rc;
  for (int d = 0; d < 3; d++) {
    if ((rc = cuda_status(cudaMemcpyAsync(h->V[d], V1[d], bytes, cudaMemcpyDeviceToDevice, h->s),
                          "sns_ns_set_state")))
      return rc;
    if ((rc = cuda_status(
             cudaMemcpyAsync(h->C0[d], cross0[d], bytes, cudaMemcpyDeviceToDevice, h->s),
             "sns_ns_set_state")))
      return rc;
  }
  h->stepped = false;
  h->carried = false;
  return OK;
}

int sns_ns_bootstrap(sns_ns* h, const void* const V0[3], const void* const omega0[3]) {
  if (!nonnull(h, "sns_ns_bootstrap") || !vec_ok(V0, "sns_ns_bootstrap") ||
      !vec_ok(omega0, "sns_ns_bootstrap"))
    return ERR_ARG;
  int rc;
  if (h->pl.real) {
    // bootstrap on full fields (pooled temporaries), then keep the half spectrum
    const Dims d{h->pl.nx_phys, h->pl.ny, h->pl.nz};
    const size_t bytes = esize(h->pl.prec) * (size_t)d.n();
    void* t[12] = {};
    rc = OK;
    for (int i = 0; i < 12 && !rc; i++) rc = pool_malloc(&t[i], bytes);
    if (!rc) rc = ns_bootstrap_fields(d, h->pl.prec, h->nu, h->dt, V0, omega0, t, t + 3, t + 6,
                                      h->s);
    if (!rc) rc = convert_half(h->V, t, d.nx, d.ny, d.nz, h->pl.prec, +1, h->s);
    if (!rc) rc = convert_half(h->C0, t + 3, d.nx, d.ny, d.nz, h->pl.prec, +1, h->s);
    cudaStreamSynchronize(h->s);
    for (void* p : t) pool_free(p);
    if (rc) return rc;
    h->stepped = false;
    h->carried = false;
    return OK;
  }
  const Dims d{h->pl.nx, h->pl.ny, h->pl.nz};
  rc = ns_bootstrap_fields(d, h->pl.prec, h->nu, h->dt, V0, omega0, h->V, h->C0, h->U, h->s);
  if (rc) return rc;
  h->stepped = false;
  h->carried = false;
  return OK;
}

int sns_ns_step(sns_ns* h, int nsteps) {
  if (!nonnull(h, "sns_ns_step")) return ERR_ARG;
  if (nsteps < 0) {
    set_error("sns_ns_step: negative step count");
    return ERR_ARG;
  }
  if (!h->profiling) {
    for (int t = 0; t < nsteps; t++) {
      int rc = OK;
      // a captured step of a carrying plan starts from K1's output in U:
      // make it there first if the state was set since
      if (h->pl.carry && !h->carried && h->cl.model == CLOSURE_NONE && h->use_graph &&
          h->eager_done) {
        if ((rc = ns_k1_once(h->pl, h->V, h->U, h->sync_words, h->s))) return rc;
        h->carried = true;
      }
      if (h->use_graph && h->eager_done && !h->exec) rc = capture_step(h);
      if (rc) return rc;
      if (h->exec) {
        rc = cuda_status(cudaGraphLaunch(h->exec, h->s), "sns_ns_step(graph)");
      } else {
        rc = step_on(h, h->s, nullptr);
        h->eager_done = true;
      }
      if (rc) return rc;
      h->stepped = true;
    }
    return OK;
  }
  if (h->cl.model != CLOSURE_NONE) {
    set_error("sns_ns_step: per-pass profiling covers the plain step only");
    return ERR_UNSUPPORTED;
  }
  for (int t = 0; t < nsteps; t++) {
    cudaEvent_t* ev = nullptr;
    if (h->profiling) {
      const size_t need = (size_t)(h->recorded + 1) * (kNSPasses + 1);
      while (h->events.size() < need) {
        cudaEvent_t e;
        int rc = cuda_status(cudaEventCreate(&e), "sns_ns_step(profile)");
        if (rc) return rc;
        h->events.push_back(e);
      }
      ev = &h->events[(size_t)h->recorded * (kNSPasses + 1)];
    }
    int rc = ns_step_once(h->pl, h->V, h->C0, h->U, h->stats_part, h->sync_words, h->nu, h->dt,
                          h->s, ev, h->W, &h->carried);
    if (rc) return rc;
    if (ev) h->recorded++;
    h->stepped = true;
  }
  return OK;
}

int sns_ns_profile(sns_ns* h, int enable) {
  if (!nonnull(h, "sns_ns_profile")) return ERR_ARG;
  h->profiling = enable != 0;
  h->recorded = 0;
  return OK;
}

int sns_ns_pass_times(sns_ns* h, double* total_ms, int* launches, int max) {
  if (!nonnull(h, "sns_ns_pass_times") || !nonnull(total_ms, "sns_ns_pass_times") ||
      !nonnull(launches, "sns_ns_pass_times") || max < 0)
    return ERR_ARG;
  int rc = cuda_status(cudaStreamSynchronize(h->s), "sns_ns_pass_times");
  if (rc) return rc;
  for (int p = 0; p < max; p++) {
    total_ms[p] = 0;
    launches[p] = 0;
  }
  for (int t = 0; t < h->recorded; t++) {
    cudaEvent_t* ev = &h->events[(size_t)t * (kNSPasses + 1)];
    for (int p = 0; p < h->pl.passes && p < max; p++) {
      float ms = 0;
      if ((rc = cuda_status(cudaEventElapsedTime(&ms, ev[p], ev[p + 1]), "sns_ns_pass_times")))
        return rc;
      total_ms[p] += ms;
      launches[p] += 1;
    }
  }
  return h->pl.passes;
}

int sns_ns_get_state(sns_ns* h, void* const V1[3], void* const omega1[3], void* const cross0[3]) {
  if (!nonnull(h, "sns_ns_get_state")) return ERR_ARG;
  if (h->pl.real) {
    // full spectra rebuilt by Hermitian symmetry
    const Dims d{h->pl.nx_phys, h->pl.ny, h->pl.nz};
    const size_t bytes = esize(h->pl.prec) * (size_t)d.n();
    int rc = OK;
    if (cross0 && cross0[0] && cross0[1] && cross0[2])
      rc = convert_half(cross0, h->C0, d.nx, d.ny, d.nz, h->pl.prec, -1, h->s);
    if (rc || (!omega1 && !(V1 && V1[0] && V1[1] && V1[2]))) return rc;
    void* t[3] = {};
    const bool own = !(V1 && V1[0] && V1[1] && V1[2]);
    void* const* vf = V1;
    if (own) {
      for (int i = 0; i < 3 && !rc; i++) rc = pool_malloc(&t[i], bytes);
      vf = t;
    }
    if (!rc) rc = convert_half(vf, h->V, d.nx, d.ny, d.nz, h->pl.prec, -1, h->s);
    if (!rc && omega1) {
      if (!vec_ok((const void* const*)omega1, "sns_ns_get_state")) {
        rc = ERR_ARG;
      } else {
        const void* v[3] = {vf[0], vf[1], vf[2]};
        rc = op_curl(v, omega1, d, h->pl.prec, h->s);
      }
    }
    if (own) {
      cudaStreamSynchronize(h->s);
      for (void* p : t) pool_free(p);
    }
    return rc;
  }
  const Dims d{h->pl.nx, h->pl.ny, h->pl.nz};
  const size_t bytes = esize(h->pl.prec) * (size_t)d.n();
  int rc;
  for (int i = 0; i < 3; i++) {
    if (V1 && V1[i] &&
        (rc = cuda_status(cudaMemcpyAsync(V1[i], h->V[i], bytes, cudaMemcpyDeviceToDevice, h->s),
                          "sns_ns_get_state")))
      return rc;
    if (cross0 && cross0[i] &&
        (rc = cuda_status(
             cudaMemcpyAsync(cross0[i], h->C0[i], bytes, cudaMemcpyDeviceToDevice, h->s),
             "sns_ns_get_state")))
      return rc;
  }
  if (omega1) {
    if (!vec_ok((const void* const*)omega1, "sns_ns_get_state")) return ERR_ARG;
    const void* v[3] = {h->V[0], h->V[1], h->V[2]};
    if ((rc = op_curl(v, omega1, d, h->pl.prec, h->s))) return rc;
  }
  return OK;
}

int sns_ns_check(sns_ns* h) {
  if (!nonnull(h, "sns_ns_check")) return ERR_ARG;
  const size_t err_index = xy_sync_words(h->pl.nz) - 1;
  int err = 0;
  int rc = cuda_status(cudaMemcpyAsync(&err, h->sync_words + err_index, sizeof(int),
                                       cudaMemcpyDeviceToHost, h->s),
                       "sns_ns_check");
  if (rc) return rc;
  if ((rc = cuda_status(cudaStreamSynchronize(h->s), "sns_ns_check"))) return rc;
  if (err) {
    cudaMemsetAsync(h->sync_words + err_index, 0, sizeof(int), h->s);
    set_error(err == 2 ? "sns_ns_step: the TMA-staged z pass refused a tile box (alignment or "
                         "range); results are invalid"
                       : "sns_ns_step: a bounded wait of a step pass (the xy dataflow pass or the "
                         "TMA-staged z pass) gave up; results are invalid");
    return ERR_TIMEOUT;
  }
  return OK;
}

int sns_ns_stats(sns_ns* h, double* div_avg, double* energy, double* enstrophy, double* max_div) {
  if (!nonnull(h, "sns_ns_stats")) return ERR_ARG;
  if (!h->stepped) {
    set_error("sns_ns_stats: no step has run since the state was set");
    return ERR_ARG;
  }
  int rc = sns_ns_check(h);
  if (rc) return rc;
  rc = ns_stats_final(h->stats_part,
                      h->cl.model != CLOSURE_NONE ? h->pl.sgs_blocks : h->pl.update_blocks,
                      h->stats_out, h->s);
  if (rc) return rc;
  double v[4];
  if ((rc = cuda_status(cudaMemcpyAsync(v, h->stats_out, sizeof(v), cudaMemcpyDeviceToHost, h->s),
                        "sns_ns_stats")))
    return rc;
  if ((rc = cuda_status(cudaStreamSynchronize(h->s), "sns_ns_stats"))) return rc;
  const double N = (double)h->pl.nx_phys * h->pl.ny * h->pl.nz;  // full grid
  if (div_avg) *div_avg = v[0] / N;
  if (energy) *energy = 0.5 * v[1] / (N * N);
  if (enstrophy) *enstrophy = 0.5 * v[2] / (N * N);
  if (max_div) *max_div = v[3];
  return OK;
}

int sns_ns_stats_async(sns_ns* h, double* out4) {
  if (!nonnull(h, "sns_ns_stats_async") || !nonnull(out4, "sns_ns_stats_async")) return ERR_ARG;
  if (!h->stepped) {
    set_error("sns_ns_stats_async: no step has run since the state was set");
    return ERR_ARG;
  }
  int rc = ns_stats_final(h->stats_part,
                          h->cl.model != CLOSURE_NONE ? h->pl.sgs_blocks : h->pl.update_blocks,
                          h->stats_out, h->s);
  if (rc) return rc;
  const double N = (double)h->pl.nx_phys * h->pl.ny * h->pl.nz;  // full grid
  if ((rc = ns_stats_normalise(h->stats_out, N, h->s))) return rc;
  return cuda_status(cudaMemcpyAsync(out4, h->stats_out, 4 * sizeof(double), cudaMemcpyDefault,
                                     h->s),
                     "sns_ns_stats_async");
}

int sns_ns_launches_per_step(sns_ns* h) {
  if (!nonnull(h, "sns_ns_launches_per_step")) return ERR_ARG;
  // a carrying plan skips K1 in every step but the first after a new state
  return h->cl.model != CLOSURE_NONE ? kLESLaunches : h->pl.passes - (h->pl.carry ? 1 : 0);
}

namespace {
// Tuned plans per device and box: (device, nx, ny, nz, precision, real).
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int, int>, NSPlan> g_tuned;
}  // namespace

int sns_ns_tune(sns_ns* h) {
  if (!nonnull(h, "sns_ns_tune")) return ERR_ARG;
  if (h->stepped || h->eager_done) {
    set_error("sns_ns_tune: tune a stepper before its first bootstrap, state or step");
    return ERR_ARG;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  const NSPlan& p = h->pl;
  const auto key = std::make_tuple(dev, p.nx, p.ny, p.nz, p.prec, p.real ? 1 : 0);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      // the knobs of the cached plan; the closure settings stay this stepper's
      NSPlan q = it->second;
      q.kc2 = p.kc2;
      q.sgs_klo = p.sgs_klo;
      q.sgs_kinv = p.sgs_kinv;
      if (q.update_blocks > p.update_blocks) {
        void* part = nullptr;
        int rc = pool_malloc(&part, sizeof(double) * 4 * std::max(q.update_blocks, q.sgs_blocks));
        if (rc) return rc;
        pool_free(h->stats_part);
        h->stats_part = static_cast<double*>(part);
      }
      h->pl = q;
      drop_graph(h);
      h->carried = false;
      return OK;
    }
  }
  // room for the diagnostics of every candidate width of the update pass
  const int max_blocks = std::max(std::max(p.update_blocks, p.sgs_blocks), p.nx * p.ny / 2);
  void* part = nullptr;
  int rc = pool_malloc(&part, sizeof(double) * 4 * max_blocks);
  if (rc) return rc;
  pool_free(h->stats_part);
  h->stats_part = static_cast<double*>(part);
  NSPlan q = h->pl;
  rc = ns_tune_plan(q, h->V, h->C0, h->U, h->stats_part, max_blocks, h->sync_words, h->s,
                    h->W[0] ? h->W : nullptr);
  if (rc) return rc;
  // the timing steps ran on seeded data: the stepper starts from zero fields
  for (int d = 0; d < 3; d++) {
    const size_t bytes = esize(q.prec) * (size_t)q.nx * q.ny * q.nz;
    if ((rc = cuda_status(cudaMemsetAsync(h->V[d], 0, bytes, h->s), "sns_ns_tune"))) return rc;
    if ((rc = cuda_status(cudaMemsetAsync(h->C0[d], 0, bytes, h->s), "sns_ns_tune"))) return rc;
  }
  h->pl = q;
  drop_graph(h);
  h->carried = false;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tuned[key] = q;
  return OK;
}

int sns_ns_describe(sns_ns* h, char* buf, int len) {
  if (!nonnull(h, "sns_ns_describe")) return ERR_ARG;
  const NSPlan& p = h->pl;
  const char* xy = p.use_xyc ? "cluster" : p.use_xy ? "dataflow"
                   : (p.xy_chunk > 0 && p.xy_chunk < p.nz) ? "slabs" : "separate";
  char tmp[256];
  const char* ord[3] = {"16-first", "remainder-first", "radix-8"};
  const int n = snprintf(tmp, sizeof(tmp),
                         "passes=%d xy=%s k1=%dx%d%s y=W%d/T%d/%s%s zW=%d%s xG=%d%s pf=%d%s%s",
                         h->cl.model != CLOSURE_NONE ? kLESLaunches : p.passes, xy,
                         p.k1_lines ? p.k1lW : p.k1W, p.k1_lines ? p.k1lT : p.k1G,
                         p.k1_lines ? "(lines)" : !p.k1_fused ? "(split)"
                         : p.k1_tma ? (p.k1_stages == 1 ? "(tma1)" : "(tma2)")
                         : p.k1_reload ? "(reload)" : "",
                         p.lineW, p.lineT,
                         ord[p.lineOrd % 3],
                         p.y_tma == 1 ? "(tma1)" : p.y_tma == 2 ? "(tma2)" : "", p.zW, p.z_tma ? "(tma)" : p.carry ? (p.carry_reload ? "(+K1r)" : "(+K1)") : p.z_pfself ? "(pfs)" : "", p.xG, p.x_tma ? "(tma)" : p.x_occ ? "(occ)" : "", p.pf_waves, p.real ? " real" : "",
                         p.tuned ? " tuned" : "");
  if (buf && len > 0) {
    strncpy(buf, tmp, (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return n;
}

int sns_ns_set_closure(sns_ns* h, int model, double cs_delta2, const void* mlp, double kc) {
  if (!nonnull(h, "sns_ns_set_closure")) return ERR_ARG;
  if (h->pl.real && model != SNS_CLOSURE_NONE) {
    set_error("sns_ns_set_closure: closures run on complex-field steppers only");
    return ERR_UNSUPPORTED;
  }
  if (!(kc >= 0)) {
    set_error("sns_ns_set_closure: the cutoff must be >= 0 (0: none)");
    return ERR_ARG;
  }
  if (model != SNS_CLOSURE_NONE && model != SNS_CLOSURE_SMAGORINSKY && model != SNS_CLOSURE_MLP) {
    set_error("sns_ns_set_closure: unknown model");
    return ERR_ARG;
  }
  if (model == SNS_CLOSURE_MLP && !mlp) {
    set_error("sns_ns_set_closure: the MLP model needs packed weights");
    return ERR_ARG;
  }
  if (model == SNS_CLOSURE_SMAGORINSKY && !(cs_delta2 >= 0)) {
    set_error("sns_ns_set_closure: (Cs Delta)^2 must be >= 0");
    return ERR_ARG;
  }
  if (model != SNS_CLOSURE_NONE && !h->U2[0]) {
    const size_t bytes = esize(h->pl.prec) * (size_t)h->pl.nx * h->pl.ny * h->pl.nz;
    for (int i = 0; i < 6; i++) {
      int rc = pool_malloc(&h->U2[i], bytes);
      if (rc) {
        for (int j = 0; j < i; j++) {
          pool_free(h->U2[j]);
          h->U2[j] = nullptr;
        }
        return rc;
      }
    }
  }
  h->cl.model = model;
  h->cl.csd2 = cs_delta2;
  h->cl.mlp = mlp;
  h->pl.kc2 = kc > 0 ? kc * kc : 1e300;
  drop_graph(h);
  h->carried = false;
  h->eager_done = false;
  return OK;
}

int sns_ns_set_sgs_band(sns_ns* h, double k_lo, double k_hi) {
  if (!nonnull(h, "sns_ns_set_sgs_band")) return ERR_ARG;
  if (!(k_lo >= 0) || !(k_hi >= 0)) {
    set_error("sns_ns_set_sgs_band: k_lo and k_hi must be >= 0");
    return ERR_ARG;
  }
  h->pl.sgs_klo = k_lo;
  h->pl.sgs_kinv = k_hi > k_lo ? 1.0 / (k_hi - k_lo) : 1e30;
  drop_graph(h);
  h->carried = false;
  h->eager_done = false;
  return OK;
}

}  // extern "C"
