// Fused pseudo-spectral Navier-Stokes step (exec/ns.cpp:167-217).
//
// State: V (Fourier velocity, 3 fields) and C0 (Fourier V x omega of the
// previous step, 3 fields); work: U (6 fields).  One step is five passes:
//
//   K1  z-inverse of (V, i k x V): the curl is formed while the tile loads
//       (ns.cpp:206 + Vector::cross's inverse copies, src/Vector.cpp:74-77)
//   K2  y-inverse of the 6 fields
//   K3  x-inverse, 1/N^2-scaled complex cross product u x omega, x-forward
//       (src/Vector.cpp:79-89), 6 fields in, 3 out
//   K4  y-forward of the 3 fields
//   K5  z-forward + Nyquist zeroing (cross1 complete), then per mode the AB2 /
//       projection / Crank-Nicolson update (ns.cpp:170-187) written over V,
//       cross1 written over C0, FP64 diagnostics (ns.cpp:206-210)
//
// The reference runs 9 separate 3D FFTs plus ~25 eager field sweeps and 15
// deep copies per step; here the history copies (ns.cpp:213-217) are
// in-place updates and every intermediate lives in U.
#include <math.h>
#include <stdlib.h>

#include <vector>

#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_ns.cuh"
#include "sns_ops.cuh"

namespace sns {

// ---------------------------------------------------------------------------
// K3: x lines -- inverse 6 fields, cross product, forward 3 fields.
template <typename T, int L>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_xcross(FieldPtrs f, const cx_t<T>* __restrict__ tw, int G, T scale2) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL, RS = row_stride(L);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const int64_t row0 = (int64_t)blockIdx.x * G;
  const int per = G * L;

  // thread t owns line t / TPL (field-major: field = line / G, row = line % G)
  // at positions j + e*TPL; loads go straight to registers, E per thread
  const int j = threadIdx.x % TPL, line = threadIdx.x / TPL;
  const int fld = line / G, gl = line - fld * G;
  C* row = sm + line * RS;
  C v[E];
  {
    const C* __restrict__ src = reinterpret_cast<const C*>(f.in[fld]);
    const int64_t i0 = (row0 + gl) * L + j;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[i0 + TPL * e];
  }
  line_fft<L>(v, row, j, tw, (T)1);
#pragma unroll
  for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
  __syncthreads();

  // c = (u/N) x (omega/N): u in rows of fields 0..2, omega in 3..5
  for (int q = threadIdx.x; q < per; q += blockDim.x) {
    const int g = q / L, p = q & (L - 1);
    C u[3], w[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      u[d] = sm[(d * G + g) * RS + pad_pos(p)];
      w[d] = sm[((3 + d) * G + g) * RS + pad_pos(p)];
    }
    const C c0 = csub(cmul(u[1], w[2]), cmul(u[2], w[1]));
    const C c1 = csub(cmul(u[2], w[0]), cmul(u[0], w[2]));
    const C c2 = csub(cmul(u[0], w[1]), cmul(u[1], w[0]));
    sm[(0 * G + g) * RS + pad_pos(p)] = cscale(scale2, c0);
    sm[(1 * G + g) * RS + pad_pos(p)] = cscale(scale2, c1);
    sm[(2 * G + g) * RS + pad_pos(p)] = cscale(scale2, c2);
  }
  __syncthreads();

  // forward x of the three products.  Lines of up to 32 threads synchronise
  // within their warp, so warps that hold only omega rows (every warp when G
  // is a multiple of the lines per warp) skip it; longer lines synchronise the
  // block and every thread takes part.
  constexpr int kLinesPerWarp = TPL <= 32 ? 32 / TPL : 1;
  const bool skip = (TPL <= 32) && (G % kLinesPerWarp == 0) && fld >= 3;
  if (!skip) {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = row[pad_pos(j + TPL * e)];
    line_sync<TPL>();
    line_fft<L>(v, row, j, tw, (T)-1);
  }

  if (fld < 3) {
    C* __restrict__ dst = reinterpret_cast<C*>(f.out[fld]);
    const int64_t i0 = (row0 + gl) * L + j;
#pragma unroll
    for (int e = 0; e < E; e++) dst[i0 + TPL * e] = v[e];
  }
}

// ---------------------------------------------------------------------------
// K5: z lines -- forward 3 fields + Nyquist zeroing, then the AB2 /
// projection / CN update per mode.
struct UpdateArgs {
  const void* U[3];  // cross1 after x, y forward passes
  void* V[3];        // in: V1, out: V (new)
  void* C0[3];       // in: cross0, out: cross1
  int nx, ny, nz;
  int W;
  double hK;      // K/2
  double nuhK;    // nu*K/2
  double* stats;  // per block: sum|div|, sum|V|^2, sum|k x V|^2, max|div|
};

template <typename T, int L>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_zfwd_update(const UpdateArgs a, const cx_t<T>* __restrict__ tw) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL, RS = row_stride(L);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  __shared__ double red[4][32];

  const int W = a.W;
  const int tiles_x = a.nx / W;
  const int x0 = (blockIdx.x % tiles_x) * W;
  const int y = blockIdx.x / tiles_x;
  const int64_t nxy = (int64_t)a.nx * a.ny;
  const int64_t base = x0 + (int64_t)a.nx * y;
  const int per = W * L;

  // thread t owns z line (field, x0 + w) at positions j + e*TPL with
  // w = t mod W, j = (t / W) mod TPL, field = t / (W*TPL): consecutive threads
  // load adjacent x, so the direct loads are coalesced
  {
    const int w = threadIdx.x % W, s = threadIdx.x / W;
    const int j = s % TPL, fld = s / TPL;
    C* row = sm + (fld * W + w) * RS;
    const C* __restrict__ src = reinterpret_cast<const C*>(a.U[fld]);
    const int64_t i0 = base + w + nxy * j;
    C v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[i0 + nxy * (TPL * e)];
    line_fft<L, true>(v, row, j, tw, (T)-1);
#pragma unroll
    for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
  }
  __syncthreads();

  const T hK = (T)a.hK, nuhK = (T)a.nuhK;
  const T ky = (T)freq_i(y, a.ny);
  const bool ynyq = (y == (a.ny >> 1));
  double s_div = 0, s_e = 0, s_w = 0, m_div = 0;
  C* __restrict__ Vp[3] = {reinterpret_cast<C*>(a.V[0]), reinterpret_cast<C*>(a.V[1]),
                           reinterpret_cast<C*>(a.V[2])};
  C* __restrict__ Cp[3] = {reinterpret_cast<C*>(a.C0[0]), reinterpret_cast<C*>(a.C0[1]),
                           reinterpret_cast<C*>(a.C0[2])};
  auto update_point = [&](int q, const C (&V1)[3], const C (&c0)[3]) {
    const int w = q % W, z = q / W;
    const int x = x0 + w;
    const int64_t idx = base + w + nxy * z;
    const T kx = (T)freq_i(x, a.nx), kz = (T)freq_i(z, a.nz);
    const bool nyq = ynyq || x == (a.nx >> 1) || z == (a.nz >> 1);
    C c1[3];
#pragma unroll
    for (int d = 0; d < 3; d++) c1[d] = nyq ? mk((T)0, (T)0) : sm[(d * W + w) * RS + pad_pos(z)];
    const T kk[3] = {kx, ky, kz};
    const T k2 = kx * kx + ky * ky + kz * kz;
    const double k2d = (double)kx * kx + (double)ky * ky + (double)kz * kz;
    // F = K/2 (3 c1 - c0)                      (ns.cpp:171)
    // lap1 = nu K/2 (-|k|^2 V1)                (ns.cpp:174)
    // s = V1 + lap1 + F; G = div s / (-|k|^2)  (ns.cpp:177-178)
    C F[3], lap[3], s[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      F[d] = cscale(hK, csub(cscale((T)3, c1[d]), c0[d]));
      lap[d] = cscale(nuhK, cscale(-k2, V1[d]));
      s[d] = cadd(cadd(V1[d], lap[d]), F[d]);
    }
    C G = cadd(cadd(ikmul(kx, s[0]), ikmul(ky, s[1])), ikmul(kz, s[2]));
    // The divisors -|k|^2 (projection) and 1 + nu K/2 |k|^2 (Crank-Nicolson)
    // are formed in FP64.  complex128 divides as the reference does; complex64
    // multiplies by the FP64 reciprocals rounded once to FP32.
    const bool nonzero = k2d != 0.0;
    const double den_cn = 1.0 + a.nuhK * k2d;
    T r_p = (T)1, r_cn = (T)1;
    if constexpr (sizeof(T) == 4) {
      if (nonzero) {
        r_p = (T)(-1.0 / k2d);
        r_cn = (T)(1.0 / den_cn);
      }
      G = cscale(r_p, G);
    } else {
      if (nonzero) G = mk(G.x / -k2d, G.y / -k2d);
    }
    // Vhalf = V1 + F - grad G; V = (Vhalf + lap1) / (1 + nu K/2 |k|^2)  (ns.cpp:181-187)
    C Vn[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      C vh = csub(cadd(V1[d], F[d]), ikmul(kk[d], G));
      C vv = cadd(vh, lap[d]);
      if constexpr (sizeof(T) == 4) {
        vv = cscale(r_cn, vv);
      } else {
        if (nonzero) vv = mk(vv.x / den_cn, vv.y / den_cn);
      }
      Vn[d] = vv;
      Vp[d][idx] = vv;
      Cp[d][idx] = c1[d];
    }
    // diagnostics of the new velocity: per-mode terms in T, sums in FP64
    const C dv = cadd(cadd(ikmul(kx, Vn[0]), ikmul(ky, Vn[1])), ikmul(kz, Vn[2]));
    const double ad = (double)sqrt(dv.x * dv.x + dv.y * dv.y);
    s_div += ad;
    m_div = fmax(m_div, ad);
    T e2 = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) e2 += Vn[d].x * Vn[d].x + Vn[d].y * Vn[d].y;
    const C om0 = csub(ikmul(ky, Vn[2]), ikmul(kz, Vn[1]));
    const C om1 = csub(ikmul(kz, Vn[0]), ikmul(kx, Vn[2]));
    const C om2 = csub(ikmul(kx, Vn[1]), ikmul(ky, Vn[0]));
    const T w2 = om0.x * om0.x + om0.y * om0.y + om1.x * om1.x + om1.y * om1.y +
                 om2.x * om2.x + om2.y * om2.y;
    s_e += (double)e2;
    s_w += (double)w2;
  };
  // two points per iteration: the 12 global loads of both are issued first
  for (int q0 = threadIdx.x; q0 < per; q0 += 2 * blockDim.x) {
    const int q1 = q0 + blockDim.x;
    const bool has1 = q1 < per;
    C V1a[3], c0a[3], V1b[3], c0b[3];
    const int64_t ia = base + (q0 % W) + nxy * (q0 / W);
    const int64_t ib = has1 ? base + (q1 % W) + nxy * (q1 / W) : ia;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      V1a[d] = Vp[d][ia];
      c0a[d] = Cp[d][ia];
      V1b[d] = Vp[d][ib];
      c0b[d] = Cp[d][ib];
    }
    update_point(q0, V1a, c0a);
    if (has1) update_point(q1, V1b, c0b);
  }
  // block reduction of the diagnostics
  for (int o = 16; o > 0; o >>= 1) {
    s_div += __shfl_xor_sync(0xffffffffu, s_div, o);
    s_e += __shfl_xor_sync(0xffffffffu, s_e, o);
    s_w += __shfl_xor_sync(0xffffffffu, s_w, o);
    m_div = fmax(m_div, __shfl_xor_sync(0xffffffffu, m_div, o));
  }
  const int warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][warp] = s_div;
    red[1][warp] = s_e;
    red[2][warp] = s_w;
    red[3][warp] = m_div;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0, t1 = 0, t2 = 0, t3 = 0;
    for (int i = 0; i < nwarps; i++) {
      t0 += red[0][i];
      t1 += red[1][i];
      t2 += red[2][i];
      t3 = fmax(t3, red[3][i]);
    }
    double* out = a.stats + 4 * (int64_t)blockIdx.x;
    out[0] = t0;
    out[1] = t1;
    out[2] = t2;
    out[3] = t3;
  }
}

__global__ void k_stats_final(const double* part, int blocks, double* out) {
  __shared__ double sm[4][256];
  double a = 0, b = 0, c = 0, m = 0;
  for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
    a += part[4 * i];
    b += part[4 * i + 1];
    c += part[4 * i + 2];
    m = fmax(m, part[4 * i + 3]);
  }
  sm[0][threadIdx.x] = a;
  sm[1][threadIdx.x] = b;
  sm[2][threadIdx.x] = c;
  sm[3][threadIdx.x] = m;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sm[0][threadIdx.x] += sm[0][threadIdx.x + o];
      sm[1][threadIdx.x] += sm[1][threadIdx.x + o];
      sm[2][threadIdx.x] += sm[2][threadIdx.x + o];
      sm[3][threadIdx.x] = fmax(sm[3][threadIdx.x], sm[3][threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) out[k] = sm[k][0];
}

// ---------------------------------------------------------------------------
// host side

namespace {

template <typename T, int L>
int launch_xcross(const NSPlan& pl, const FieldPtrs& f, int64_t rows, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  const int G = pl.xG;
  const int threads = 6 * G * TPL;
  const size_t smem = (size_t)6 * G * row_stride(L) * sizeof(C);
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_xcross<T, L>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_xcross)");
    attr[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  const double N = (double)pl.nx * pl.ny * pl.nz;
  const int blocks = (int)(rows / G);
  k_xcross<T, L><<<blocks, threads, smem, s>>>(f, tw, G, (T)(1.0 / (N * N)));
  SNS_CHECK_LAUNCH("k_xcross");
  return OK;
}

template <typename T, int L>
int launch_update(const NSPlan& pl, const UpdateArgs& a, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  const int threads = 3 * a.W * TPL;
  const size_t smem = (size_t)3 * a.W * row_stride(L) * sizeof(C);
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_zfwd_update<T, L>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_zfwd_update)");
    attr[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  k_zfwd_update<T, L><<<pl.update_blocks, threads, smem, s>>>(a, tw);
  SNS_CHECK_LAUNCH("k_zfwd_update");
  return OK;
}

template <typename T>
int xcross(const NSPlan& pl, const FieldPtrs& f, int64_t rows, cudaStream_t s) {
  switch (pl.nx) {
    case 4: return launch_xcross<T, 4>(pl, f, rows, s);
    case 8: return launch_xcross<T, 8>(pl, f, rows, s);
    case 16: return launch_xcross<T, 16>(pl, f, rows, s);
    case 32: return launch_xcross<T, 32>(pl, f, rows, s);
    case 64: return launch_xcross<T, 64>(pl, f, rows, s);
    case 128: return launch_xcross<T, 128>(pl, f, rows, s);
    case 256: return launch_xcross<T, 256>(pl, f, rows, s);
    case 512: return launch_xcross<T, 512>(pl, f, rows, s);
    case 1024: return launch_xcross<T, 1024>(pl, f, rows, s);
    default: set_error("fused NS step: nx must be a power of two in [4, 1024]"); return ERR_UNSUPPORTED;
  }
}

template <typename T>
int update(const NSPlan& pl, const UpdateArgs& a, cudaStream_t s) {
  switch (pl.nz) {
    case 4: return launch_update<T, 4>(pl, a, s);
    case 8: return launch_update<T, 8>(pl, a, s);
    case 16: return launch_update<T, 16>(pl, a, s);
    case 32: return launch_update<T, 32>(pl, a, s);
    case 64: return launch_update<T, 64>(pl, a, s);
    case 128: return launch_update<T, 128>(pl, a, s);
    case 256: return launch_update<T, 256>(pl, a, s);
    case 512: return launch_update<T, 512>(pl, a, s);
    case 1024: return launch_update<T, 1024>(pl, a, s);
    default: set_error("fused NS step: nz must be a power of two in [4, 1024]"); return ERR_UNSUPPORTED;
  }
}

int elems(int L) { return L >= 16 ? 16 : L; }

}  // namespace

int ns_plan(NSPlan& pl, int nx, int ny, int nz, int prec) {
  pl = NSPlan{};
  pl.nx = nx;
  pl.ny = ny;
  pl.nz = nz;
  pl.prec = prec;
  for (int n : {nx, ny, nz})
    if (!is_pow2(n) || n < 4 || n > 1024) {
      set_error("fused NS step: dimensions must be powers of two in [4, 1024]");
      return ERR_UNSUPPORTED;
    }
  const size_t esz = prec == PREC_C128 ? 16 : 8;
  // K3 tile: G rows of all six fields
  {
    const int TPL = nx / elems(nx);
    int G = 1;
    while (6 * (G * 2) * TPL <= 384 && ((int64_t)ny * nz) % (G * 2) == 0 &&
           (size_t)6 * G * 2 * row_stride(nx) * esz <= 110 * 1024)
      G *= 2;
    if (6 * G * TPL > max_threads(prec)) {
      set_error("fused NS step: nx too large for the x-pass tile");
      return ERR_UNSUPPORTED;
    }
    pl.xG = G;
  }
  // K5 tile: W adjacent z lines of three fields
  {
    const int TPL = nz / elems(nz);
    int W = 1;
    int Wmax = prec == PREC_C128 ? 8 : 16;
    // tile width override for tuning sweeps (SNS_Z_W, a power of two)
    if (const char* e = getenv("SNS_Z_W")) {
      const int v = atoi(e);
      if (v >= 1 && (v & (v - 1)) == 0) Wmax = v;
    }
    while (W * 2 <= Wmax && nx % (W * 2) == 0 && 3 * (W * 2) * TPL <= max_threads(prec) &&
           (size_t)3 * W * 2 * row_stride(nz) * esz <= 110 * 1024)
      W *= 2;
    pl.zW = W;
    pl.update_blocks = (nx / W) * ny;
  }
  // xy phase: three separate full-domain passes by default.  SNS_XY_PASSES=1
  // selects the persistent dataflow launch (sns_xy.cu), which moves a third of
  // the HBM bytes of the separate passes but measured slower on B200 at 256^3
  // (1.09 vs 0.79 ms): these passes are bound by issue and latency, not HBM.
  const char* env = getenv("SNS_XY_PASSES");
  const bool dataflow = env && env[0] == '1';
  pl.use_xy = dataflow && xy_supported(nx, ny, prec) && xy_plan(pl.xy, nx, ny, nz, prec) == OK;
  // separate passes run in slabs of xy_chunk planes (SNS_XY_CHUNK; 0 = one slab)
  pl.xy_chunk = 0;
  if (const char* e = getenv("SNS_XY_CHUNK")) pl.xy_chunk = atoi(e);
  pl.passes = (pl.use_xy || (pl.xy_chunk > 0 && pl.xy_chunk < nz)) ? 3 : 5;
  return OK;
}

int ns_step_once(const NSPlan& pl, void* const V[3], void* const C0[3], void* const U[6],
                 double* stats, int* sync_words, double nu, double dt, cudaStream_t s,
                 cudaEvent_t* ev) {
  const int nx = pl.nx, ny = pl.ny, nz = pl.nz, prec = pl.prec;
  int rc;
  int pass = 0;
  auto mark = [&]() {
    if (ev) cudaEventRecord(ev[pass], s);
    pass++;
  };
  mark();
  // K1: z-inverse of (V, i k x V)
  {
    FieldPtrs f{};
    f.n = 6;
    for (int d = 0; d < 3; d++) f.in[d] = V[d];
    for (int i = 0; i < 6; i++) f.out[i] = U[i];
    LineGeo g = axis_geo(2, nx, ny, nz, prec);
    if ((rc = run_line_pass(g, f, +1, 0, 1.0, prec, s, PRO_CURL6))) return rc;
    mark();
  }
  if (pl.use_xy) {
    // K2 + K3 + K4 as one persistent dataflow launch (sns_xy.cu)
    if ((rc = xy_run(pl.xy, U, sync_words, s))) return rc;
    mark();
  }
  // K2, K3, K4 on the planes [z0, z0 + pz): the passes treat the slab as an
  // nx*ny*pz field at an offset pointer (the 1/N^2 scale keeps the full N)
  const size_t esz = prec == PREC_C128 ? 16 : 8;
  auto xy_range = [&](int z0, int pz, bool marks) -> int {
    const size_t off = esz * (size_t)z0 * nx * ny;
    void* Uc[6];
    for (int i = 0; i < 6; i++) Uc[i] = static_cast<char*>(U[i]) + off;
    {  // K2: y-inverse of the six fields
      FieldPtrs f{};
      f.n = 6;
      for (int i = 0; i < 6; i++) f.in[i] = f.out[i] = Uc[i];
      LineGeo g = axis_geo(1, nx, ny, pz, prec);
      int r = run_line_pass(g, f, +1, 0, 1.0, prec, s);
      if (r) return r;
      if (marks) mark();
    }
    {  // K3: x-inverse, cross product, x-forward
      FieldPtrs f{};
      f.n = 6;
      for (int i = 0; i < 6; i++) f.in[i] = Uc[i];
      for (int i = 0; i < 3; i++) f.out[i] = Uc[i];
      const int64_t rows = (int64_t)ny * pz;
      int r = prec == PREC_C128 ? xcross<double>(pl, f, rows, s) : xcross<float>(pl, f, rows, s);
      if (r) return r;
      if (marks) mark();
    }
    {  // K4: y-forward of the cross product
      FieldPtrs f{};
      f.n = 3;
      for (int i = 0; i < 3; i++) f.in[i] = f.out[i] = Uc[i];
      LineGeo g = axis_geo(1, nx, ny, pz, prec);
      int r = run_line_pass(g, f, -1, 0, 1.0, prec, s);
      if (r) return r;
    }
    return OK;
  };
  if (!pl.use_xy) {
    if (pl.xy_chunk > 0 && pl.xy_chunk < nz) {
      // slabs of xy_chunk planes, so each slab's intermediates stay in L2
      for (int z0 = 0; z0 < nz; z0 += pl.xy_chunk)
        if ((rc = xy_range(z0, std::min(pl.xy_chunk, nz - z0), false))) return rc;
    } else if ((rc = xy_range(0, nz, true))) {
      return rc;
    }
    mark();
  }
  // K5: z-forward + Nyquist zeroing + AB2/projection/CN update
  {
    UpdateArgs a{};
    for (int d = 0; d < 3; d++) {
      a.U[d] = U[d];
      a.V[d] = V[d];
      a.C0[d] = C0[d];
    }
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.W = pl.zW;
    a.hK = dt / 2;
    a.nuhK = nu * dt / 2;
    a.stats = stats;
    rc = prec == PREC_C128 ? update<double>(pl, a, s) : update<float>(pl, a, s);
    if (rc) return rc;
    mark();
  }
  return OK;
}

int ns_stats_final(const NSPlan& pl, const double* partials, double* out4, cudaStream_t s) {
  k_stats_final<<<1, 256, 0, s>>>(partials, pl.update_blocks, out4);
  SNS_CHECK_LAUNCH("k_stats_final");
  return OK;
}

}  // namespace sns
