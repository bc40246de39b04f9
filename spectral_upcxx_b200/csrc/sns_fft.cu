// Batched line-FFT passes: the replacement for FFT1D's per-line FFTW calls
// (src/FFT1D.cpp:95-101) and for the three 1D phases of Scalar::transform
// (src/Scalar.cpp:419-566).  One kernel launch transforms every line along
// one axis of up to twelve fields.  A CTA owns a tile of W adjacent lines x G
// groups: its threads load the tile straight into registers with coalesced
// reads, run the register/shared-memory Stockham line FFT, and store the
// tile back with the epilogue (1/N scaling, Nyquist zeroing) applied.  Tiles
// are disjoint, so passes run in place; the reference's transpose buffer
// (`tmp`, src/Scalar.cpp:113-122) is not needed.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_tiles.cuh"
#include "sns_ens.cuh"

namespace sns {

bool is_pow2(int64_t n) { return n >= 1 && (n & (n - 1)) == 0; }
bool line_supported(int64_t L) { return L == 1 || (is_pow2(L) && L <= kMaxLine); }

void twiddle_host_table(int L, int prec, std::vector<unsigned char>& out) {
  std::vector<double> tab(2 * (size_t)L);
  for (int m = 0; m < L; m++) {
    double c, s;
    cis_octant(m, L, &c, &s);
    tab[2 * m] = c;
    tab[2 * m + 1] = -s;  // exp(-i 2 pi m / L)
  }
  if (prec == PREC_C128) {
    out.resize(sizeof(double) * tab.size());
    memcpy(out.data(), tab.data(), out.size());
  } else {
    std::vector<float> f(tab.size());
    for (size_t i = 0; i < tab.size(); i++) f[i] = (float)tab[i];
    out.resize(sizeof(float) * f.size());
    memcpy(out.data(), f.data(), out.size());
  }
}

const void* twiddles(int L, int prec) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, void*> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_tuple(dev, L, prec);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  std::vector<unsigned char> tab;
  twiddle_host_table(L, prec, tab);
  void* d = nullptr;
  if (cudaMalloc(&d, tab.size()) != cudaSuccess) return nullptr;
  cudaMemcpy(d, tab.data(), tab.size(), cudaMemcpyHostToDevice);
  cache[key] = d;
  return d;
}

// One CTA per (field, tile); the tile body is in sns_tiles.cuh.
template <typename T, int L, int PRO, int ORD = RADIX16_FIRST>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_line_pass(const LineGeo geo, const FieldPtrs f, const cx_t<T>* __restrict__ tw, T sg,
                T scale, int flags, int wshift) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_trigger();
  pdl_wait();
  line_pass_tile<T, L, PRO, ParamFields, ORD>(geo, ParamFields{f}, f.n, tw, sg, scale, flags,
                                               wshift, (int64_t)blockIdx.x,
                                               reinterpret_cast<cx_t<T>*>(smem_raw));
}

// epilogue-only pass (used when every axis has length 1)
template <typename T>
__global__ void k_scale_zero(const FieldPtrs f, int64_t n, int nx, int ny, int nz, T scale,
                             int flags) {
  using C = cx_t<T>;
  const int field = blockIdx.y;
  C* d = reinterpret_cast<C*>(f.out[field]);
  const C* s = reinterpret_cast<const C*>(f.in[field]);
  const int64_t nxy = (int64_t)nx * ny;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    C v = s[i];
    if (flags & PASS_SCALE) v = cscale(scale, v);
    if (flags & PASS_ZERO_NYQUIST) {
      int64_t z = i / nxy, r = i - z * nxy, y = r / nx, x = r - y * nx;
      if (x == (nx >> 1) || y == (ny >> 1) || z == (nz >> 1)) v = mk((T)0, (T)0);
    }
    d[i] = v;
  }
}

template <typename T, int L, int PRO, int ORD = RADIX16_FIRST>
static int launch_pass(const LineGeo& geo, const FieldPtrs& f, int sign, int flags,
                       double scale, cudaStream_t stream) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  const int lines = geo.W * geo.G;
  const int threads = lines * TPL;
  const size_t smem = (size_t)lines * tile_stride(L, geo.W, (int)sizeof(C)) * sizeof(C);
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_line_pass<T, L, PRO, ORD>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_line_pass)");
    attr_set[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(
      geo.tw ? geo.tw : twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  int wshift = 0;
  while ((1 << wshift) < geo.W) wshift++;
  const int64_t blocks = geo.TA * geo.TB * f.n;
  if (blocks > 0x7fffffff) {
    set_error("line pass: grid too large");
    return ERR_UNSUPPORTED;
  }
  LineGeo g = geo;
  g.pf = tiles_in_waves(k_line_pass<T, L, PRO, ORD>, threads, smem, geo.pfw);
  cudaError_t e = launch_pdl(k_line_pass<T, L, PRO, ORD>, dim3((unsigned)blocks), dim3(threads),
                             smem, stream, g, f, tw, (T)sign, (T)scale, flags, wshift);
  if (e != cudaSuccess) return cuda_status(e, "k_line_pass");
  return OK;
}

// Radix orders other than RADIX16_FIRST are built for the plain-load passes
// of the line lengths where the tuner chooses among them.
template <typename T, int L, int PRO>
static int launch_ordered(const LineGeo& geo, const FieldPtrs& f, int sign, int flags,
                          double scale, cudaStream_t stream) {
  if constexpr (PRO == PRO_LOAD && L >= 64 && L <= 1024) {
    if (geo.ord == RADIX_REM_FIRST)
      return launch_pass<T, L, PRO, RADIX_REM_FIRST>(geo, f, sign, flags, scale, stream);
    if (geo.ord == RADIX8)
      return launch_pass<T, L, PRO, RADIX8>(geo, f, sign, flags, scale, stream);
  }
  return launch_pass<T, L, PRO>(geo, f, sign, flags, scale, stream);
}

template <typename T, int PRO>
static int dispatch_pass(const LineGeo& geo, const FieldPtrs& f, int sign, int flags,
                         double scale, cudaStream_t stream) {
  switch (geo.L) {
    case 2: return launch_pass<T, 2, PRO>(geo, f, sign, flags, scale, stream);
    case 4: return launch_pass<T, 4, PRO>(geo, f, sign, flags, scale, stream);
    case 8: return launch_pass<T, 8, PRO>(geo, f, sign, flags, scale, stream);
    case 16: return launch_pass<T, 16, PRO>(geo, f, sign, flags, scale, stream);
    case 32: return launch_pass<T, 32, PRO>(geo, f, sign, flags, scale, stream);
    case 64: return launch_ordered<T, 64, PRO>(geo, f, sign, flags, scale, stream);
    case 128: return launch_ordered<T, 128, PRO>(geo, f, sign, flags, scale, stream);
    case 256: return launch_ordered<T, 256, PRO>(geo, f, sign, flags, scale, stream);
    case 512: return launch_ordered<T, 512, PRO>(geo, f, sign, flags, scale, stream);
    case 1024: return launch_ordered<T, 1024, PRO>(geo, f, sign, flags, scale, stream);
    case 2048: return launch_pass<T, 2048, PRO>(geo, f, sign, flags, scale, stream);
    case 4096: return launch_pass<T, 4096, PRO>(geo, f, sign, flags, scale, stream);
    default:
      set_error("line length " + std::to_string(geo.L) +
                " is not supported (powers of two up to 4096)");
      return ERR_UNSUPPORTED;
  }
}

int run_line_pass(const LineGeo& geo, const FieldPtrs& f, int sign, int flags, double scale,
                  int prec, cudaStream_t stream, int prologue) {
  if (f.n < 1 || f.n > kMaxFields) {
    set_error("line pass: 1..12 fields");
    return ERR_ARG;
  }
  if (geo.TA * geo.TB == 0) return OK;
  if (prologue == PRO_CURL6) {
    if (f.n != 6) {
      set_error("curl prologue needs six output fields");
      return ERR_ARG;
    }
    if (prec == PREC_C128)
      return dispatch_pass<double, PRO_CURL6>(geo, f, sign, flags, scale, stream);
    return dispatch_pass<float, PRO_CURL6>(geo, f, sign, flags, scale, stream);
  }
  if (prologue == PRO_OMEGA) {
    if (f.n != 6) {
      set_error("omega prologue needs six output fields");
      return ERR_ARG;
    }
    for (int i = 0; i < 6; i++)
      if (!f.out[i] || (i < 5 && !f.in[i])) {
        set_error("line pass: null field pointer");
        return ERR_ARG;
      }
    if (prec == PREC_C128)
      return dispatch_pass<double, PRO_OMEGA>(geo, f, sign, flags, scale, stream);
    return dispatch_pass<float, PRO_OMEGA>(geo, f, sign, flags, scale, stream);
  }
  if (prologue != PRO_LOAD && prologue != PRO_IKAXIS) {
    set_error("line pass: unknown prologue");
    return ERR_ARG;
  }
  for (int i = 0; i < f.n; i++)
    if (!f.in[i] || !f.out[i]) {
      set_error("line pass: null field pointer");
      return ERR_ARG;
    }
  if (prologue == PRO_IKAXIS) {
    if (prec == PREC_C128)
      return dispatch_pass<double, PRO_IKAXIS>(geo, f, sign, flags, scale, stream);
    return dispatch_pass<float, PRO_IKAXIS>(geo, f, sign, flags, scale, stream);
  }
  if (prec == PREC_C128) return dispatch_pass<double, PRO_LOAD>(geo, f, sign, flags, scale, stream);
  return dispatch_pass<float, PRO_LOAD>(geo, f, sign, flags, scale, stream);
}

static int elems_per_thread(int L) { return L >= 16 ? 16 : L; }

// Choose W adjacent lines and G groups for a pass of line length L.
static void choose_tile(LineGeo& g, int64_t adjacent, int64_t groups, int prec, int wmax,
                        int tmax) {
  const int TPL = g.L / elems_per_thread(g.L);
  const size_t esz = prec == PREC_C128 ? 16 : 8;
  const size_t smem_cap = 200 * 1024;
  int W = 1;
  int Wmax = prec == PREC_C128 ? 8 : 16;  // 128-byte runs
  if (wmax > 0) Wmax = wmax;  // a tuned width
  // run-width override for tuning sweeps (SNS_LINE_W, a power of two)
  if (const char* e = wmax > 0 ? nullptr : getenv("SNS_LINE_W")) {
    const int v = atoi(e);
    if (v >= 1 && (v & (v - 1)) == 0) Wmax = v;
  }
  while (W * 2 <= Wmax && adjacent % (W * 2) == 0 && W * 2 * TPL <= max_threads(prec) &&
         (size_t)(W * 2) * tile_stride(g.L, W * 2, (int)esz) * esz <= smem_cap)
    W *= 2;
  int G = 1;
  const int tcap = tmax > 0 ? tmax : 256;  // threads per CTA up to which groups are added
  while (W * G * 2 * TPL <= tcap && W * G * 2 * TPL <= max_threads(prec) &&
         groups % (G * 2) == 0 &&
         (size_t)(W * G * 2) * tile_stride(g.L, W, (int)esz) * esz <= smem_cap / 2)
    G *= 2;
  g.W = W;
  g.G = G;
}

LineGeo axis_geo(int axis, int nx, int ny, int nz, int prec, int wmax, int tmax, int ord) {
  LineGeo g{};
  // radix-order override for tests and sweeps (SNS_RADIX_ORDER = 0, 1, 2)
  if (ord == 0)
    if (const char* e = getenv("SNS_RADIX_ORDER")) ord = atoi(e) % kRadixOrders;
  g.ord = ord;
  g.nx = nx;
  g.axis = axis;
  g.ny = ny;
  g.nz = nz;
  const int64_t nxy = (int64_t)nx * ny;
  if (axis == 0) {
    g.L = nx;
    g.ps = 1;
    g.gs = nx;
    choose_tile(g, 1, (int64_t)ny * nz, prec, wmax, tmax);
    g.TA = (int64_t)ny * nz / g.G;
    g.TB = 1;
    g.sa = (int64_t)g.G * nx;
    g.sb = 0;
  } else if (axis == 1) {
    g.L = ny;
    g.ps = nx;
    g.gs = nxy;
    choose_tile(g, nx, nz, prec, wmax, tmax);
    g.TA = nx / g.W;
    g.TB = nz / g.G;
    g.sa = g.W;
    g.sb = (int64_t)g.G * nxy;
  } else {
    g.L = nz;
    g.ps = nxy;
    g.gs = nx;
    choose_tile(g, nx, ny, prec, wmax, tmax);
    g.TA = nx / g.W;
    g.TB = ny / g.G;
    g.sa = g.W;
    g.sb = (int64_t)g.G * nx;
  }
  return g;
}

int fft3d(void* const* fields, int nf, int nx, int ny, int nz, int sign, int flags, int prec,
          cudaStream_t stream, const void* const* tw_axes) {
  if (nx < 1 || ny < 1 || nz < 1 || nf < 1 || nf > kMaxFields) {
    set_error("fft3d: bad dimensions or field count");
    return ERR_ARG;
  }
  if (!line_supported(nx) || !line_supported(ny) || !line_supported(nz)) {
    set_error("fft3d: dimensions must be powers of two up to 4096");
    return ERR_UNSUPPORTED;
  }
  FieldPtrs f{};
  f.n = nf;
  for (int i = 0; i < nf; i++) f.in[i] = f.out[i] = fields[i];
  const double N = (double)nx * ny * nz;
  // a tuned plan of this shape (callers that pass their own twiddle tables
  // keep the default plan and never trigger a tuning run)
  FftChoice tc{};
  bool tuned = false;
  if (!tw_axes) {
    tuned = fft3d_tuned(nx, ny, nz, nf, prec, &tc);
    if (!tuned && tune_on_first_use()) {
      int rc = fft3d_tune(nx, ny, nz, nf, prec, stream);
      if (rc) return rc;
      tuned = fft3d_tuned(nx, ny, nz, nf, prec, &tc);
    }
  }
  auto geo = [&](int axis) {
    return tuned ? axis_geo(axis, nx, ny, nz, prec, tc.wmax[axis], tc.tmax[axis], tc.ord[axis])
                 : axis_geo(axis, nx, ny, nz, prec);
  };
  // a pass of the plan: the TMA-staged form where the tuned plan chose it
  // (SNS_FFT_TMA = 1 or 2 stages asks for it on the passes of an untuned
  // plan)
  int forced = 0;
  if (const char* e = getenv("SNS_FFT_TMA")) forced = atoi(e);
  if (forced != 1 && forced != 2) forced = 0;
  int* err_word = (tuned || forced) && !tw_axes ? fft_tma_err_word() : nullptr;
  auto pass = [&](int axis, const LineGeo& g, int sg, int fl) {
    const int S = tuned ? tc.tma[axis] : forced;
    if (S && err_word && nf <= 6 && line_tma_ok(g, prec, S))
      return run_line_pass_tma(g, f, sg, fl, 1.0 / N, prec, stream, S, err_word);
    return run_line_pass(g, f, sg, fl, 1.0 / N, prec, stream);
  };
  const bool plane = tuned ? tc.plane : true;
  if (!tw_axes && plane && fft_xy_supported(nx, ny, nz, nf, prec)) {
    // two passes: xy planes and z lines (forward xy first, inverse z first),
    // the epilogue on the second
    const bool z_pass = nz > 1;
    if (sign < 0) {
      int rc = fft_xy_pass(f, nx, nz, sign, z_pass ? 0 : flags, 1.0 / N, prec, stream);
      if (rc || !z_pass) return rc;
      return pass(2, geo(2), sign, flags);
    }
    if (z_pass) {
      int rc = pass(2, geo(2), sign, 0);
      if (rc) return rc;
    }
    return fft_xy_pass(f, nx, nz, sign, flags, 1.0 / N, prec, stream);
  }
  // axes of length 1 are identities; the epilogue rides on the last real pass
  int axes[3], na = 0;
  const int order_fwd[3] = {0, 1, 2}, order_inv[3] = {2, 1, 0};
  const int* order = sign < 0 ? order_fwd : order_inv;
  const int dims[3] = {nx, ny, nz};
  for (int i = 0; i < 3; i++)
    if (dims[order[i]] > 1) axes[na++] = order[i];
  for (int i = 0; i < na; i++) {
    LineGeo g = geo(axes[i]);
    if (tw_axes) g.tw = tw_axes[axes[i]];
    int fl = (i == na - 1) ? flags : 0;
    int rc = pass(axes[i], g, sign, fl);
    if (rc) return rc;
  }
  if (na == 0 && flags) {
    const int64_t n = (int64_t)nx * ny * nz;
    dim3 grid((unsigned)((n + 255) / 256), nf);
    if (prec == PREC_C128)
      k_scale_zero<double><<<grid, 256, 0, stream>>>(f, n, nx, ny, nz, 1.0 / N, flags);
    else
      k_scale_zero<float><<<grid, 256, 0, stream>>>(f, n, nx, ny, nz, (float)(1.0 / N), flags);
    SNS_CHECK_LAUNCH("k_scale_zero");
  }
  return OK;
}

namespace {

std::mutex g_fft_tune_mu;
std::map<std::tuple<int, int, int, int, int, int>, FftChoice> g_fft_tuned;

std::tuple<int, int, int, int, int, int> fft_key(int nx, int ny, int nz, int nf, int prec) {
  int dev = 0;
  cudaGetDevice(&dev);
  return std::make_tuple(dev, nx, ny, nz, nf, prec);
}

}  // namespace

bool tune_on_first_use() {
  static const bool on = [] {
    const char* e = getenv("SNS_TUNE");
    return e && e[0] == '1';
  }();
  return on;
}

bool fft3d_tuned(int nx, int ny, int nz, int nf, int prec, FftChoice* out) {
  std::lock_guard<std::mutex> lock(g_fft_tune_mu);
  auto it = g_fft_tuned.find(fft_key(nx, ny, nz, nf, prec));
  if (it == g_fft_tuned.end()) return false;
  *out = it->second;
  return true;
}

int fft3d_tune(int nx, int ny, int nz, int nf, int prec, cudaStream_t stream) {
  if (nx < 1 || ny < 1 || nz < 1 || nf < 1 || nf > kMaxFields) {
    set_error("fft3d_tune: bad dimensions or field count");
    return ERR_ARG;
  }
  if (!line_supported(nx) || !line_supported(ny) || !line_supported(nz)) {
    set_error("fft3d_tune: dimensions must be powers of two up to 4096");
    return ERR_UNSUPPORTED;
  }
  const size_t bytes = (prec == PREC_C128 ? 16 : 8) * (size_t)nx * ny * nz;
  void* fld[kMaxFields] = {nullptr};
  int rc = OK;
  for (int i = 0; i < nf && rc == OK; i++) {
    rc = pool_malloc(&fld[i], bytes);
    if (rc == OK) rc = cuda_status(cudaMemsetAsync(fld[i], 0, bytes, stream), "fft3d_tune");
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (rc == OK) rc = cuda_status(cudaEventCreate(&e0), "fft3d_tune");
  if (rc == OK) rc = cuda_status(cudaEventCreate(&e1), "fft3d_tune");
  FieldPtrs f{};
  f.n = nf;
  for (int i = 0; i < nf; i++) f.in[i] = f.out[i] = fld[i];
  // least time of `reps` forward + inverse applications of a launch sequence
  auto timed = [&](auto&& launch, float* out) -> int {
    float best = 3.4e38f;
    for (int r = 0; r < 4; r++) {
      int e = cuda_status(cudaEventRecord(e0, stream), "fft3d_tune");
      if (!e) e = launch(-1);
      if (!e) e = launch(+1);
      if (!e) e = cuda_status(cudaEventRecord(e1, stream), "fft3d_tune");
      if (!e) e = cuda_status(cudaEventSynchronize(e1), "fft3d_tune");
      if (e) return e;
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      if (r) best = std::min(best, t);  // the first run sets the kernels up
    }
    *out = best;
    return OK;
  };
  FftChoice c{};
  for (int a = 0; a < 3; a++) {
    c.wmax[a] = 0;
    c.tmax[a] = 0;
    c.ord[a] = 0;
    c.tma[a] = 0;
  }
  c.plane = false;
  const int dims[3] = {nx, ny, nz};
  // the pass of axis a under a candidate plan (its TMA-staged form if chosen)
  int* err_word = fft_tma_err_word();
  auto tma_fits = [&](const FftChoice& q, int a, int S) {
    return S == 0 || (err_word && nf <= 6 &&
                      line_tma_ok(axis_geo(a, nx, ny, nz, prec, q.wmax[a], q.tmax[a], q.ord[a]),
                                  prec, S));
  };
  auto one = [&](const FftChoice& q, int a, int sg) {
    const LineGeo g = axis_geo(a, nx, ny, nz, prec, q.wmax[a], q.tmax[a], q.ord[a]);
    if (q.tma[a] && tma_fits(q, a, q.tma[a]))
      return run_line_pass_tma(g, f, sg, 0, 1.0, prec, stream, q.tma[a], err_word);
    return run_line_pass(g, f, sg, 0, 1.0, prec, stream);
  };
  for (int a = 0; a < 3 && rc == OK; a++) {
    if (dims[a] < 2) continue;
    // run width (y, z) and thread cap, then radix order, of this axis's pass
    float best = 3.4e38f;
    FftChoice bc = c;
    for (int W : {4, 8, 16, 32})
      for (int T : {128, 256, 512})
        for (int S = 0; S <= 2 && rc == OK; S++) {
          if (a == 0 && W != 16) continue;  // x lines are single lines
          FftChoice q = c;
          q.wmax[a] = W;
          q.tmax[a] = T;
          q.tma[a] = S;
          if (!tma_fits(q, a, S)) continue;
          float t = 0;
          rc = timed([&](int sg) { return one(q, a, sg); }, &t);
          if (rc) break;
          if (getenv("SNS_TUNE_LOG") && getenv("SNS_TUNE_LOG")[0] == '1')
            fprintf(stderr, "fft3d_tune axis=%d W=%d T=%d tma=%d ms=%.4f\n", a, W, T, S, t);
          if (t < best) {
            best = t;
            bc = q;
          }
        }
    c = bc;
    if (rc == OK && dims[a] >= 64 && dims[a] <= 1024) {
      for (int o = 1; o < kRadixOrders && rc == OK; o++) {
        FftChoice q = c;
        q.ord[a] = o;
        if (!tma_fits(q, a, q.tma[a])) continue;
        float t = 0;
        rc = timed([&](int sg) { return one(q, a, sg); }, &t);
        if (rc == OK && t < best) {
          best = t;
          bc = q;
        }
      }
      c = bc;
    }
  }
  // the xy plane pass against the tuned x and y line passes
  if (rc == OK && fft_xy_supported(nx, ny, nz, nf, prec)) {
    float t_lines = 0, t_plane = 0;
    rc = timed([&](int sg) {
      int e = one(c, 0, sg);
      if (!e) e = one(c, 1, sg);
      return e;
    }, &t_lines);
    if (rc == OK)
      rc = timed([&](int sg) { return fft_xy_pass(f, nx, nz, sg, 0, 1.0, prec, stream); },
                 &t_plane);
    c.plane = rc == OK && t_plane < t_lines;
  }
  // keep the tuned plan only if the whole transform pair beats the default
  // plan's (pass-by-pass timings of L2-resident fields can mislead)
  if (rc == OK) {
    auto whole = [&](const FftChoice* ch, float* t) {
      return timed([&](int sg) -> int {
        const int axes_fwd[3] = {0, 1, 2}, axes_inv[3] = {2, 1, 0};
        const int* order = sg < 0 ? axes_fwd : axes_inv;
        const bool plane = ch ? ch->plane : true;
        if (plane && fft_xy_supported(nx, ny, nz, nf, prec)) {
          auto zpass = [&]() {
            return ch ? one(*ch, 2, sg)
                      : run_line_pass(axis_geo(2, nx, ny, nz, prec), f, sg, 0, 1.0, prec, stream);
          };
          int e = 0;
          if (sg < 0) {
            e = fft_xy_pass(f, nx, nz, sg, 0, 1.0, prec, stream);
            if (!e && nz > 1) e = zpass();
          } else {
            if (nz > 1) e = zpass();
            if (!e) e = fft_xy_pass(f, nx, nz, sg, 0, 1.0, prec, stream);
          }
          return e;
        }
        for (int i = 0; i < 3; i++) {
          const int a = order[i];
          if (dims[a] < 2) continue;
          int e = ch ? one(*ch, a, sg)
                     : run_line_pass(axis_geo(a, nx, ny, nz, prec), f, sg, 0, 1.0, prec, stream);
          if (e) return e;
        }
        return OK;
      }, t);
    };
    float t_default = 0, t_tuned = 0;
    rc = whole(nullptr, &t_default);
    if (rc == OK) rc = whole(&c, &t_tuned);
    if (rc == OK && t_default <= t_tuned) {
      for (int a = 0; a < 3; a++) {
        c.wmax[a] = 0;
        c.tmax[a] = 0;
        c.ord[a] = 0;
        c.tma[a] = 0;
      }
      c.plane = true;
    }
  }
  // a TMA-staged candidate that recorded a failure must not be kept
  if (rc == OK) rc = fft_tma_check(stream);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  for (int i = 0; i < nf; i++) pool_free(fld[i]);
  if (rc) return rc;
  std::lock_guard<std::mutex> lock(g_fft_tune_mu);
  g_fft_tuned[fft_key(nx, ny, nz, nf, prec)] = c;
  return OK;
}

}  // namespace sns
