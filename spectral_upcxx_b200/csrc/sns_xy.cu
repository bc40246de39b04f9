// The xy phase of the fused NS step as one persistent dataflow kernel.
//
// Per step the y-inverse of the six fields (K2), the x cross pass (K3) and the
// y-forward of the three cross-product fields (K4) touch one z plane at a time.
// Run as three full-domain kernels they stream 27 field-passes through HBM;
// here they run as work items of one launch, ordered plane by plane so that a
// plane's intermediates are consumed from L2 soon after they are produced:
//
//   A(z, f, xt)  y-inverse of field f (0..5) on x columns xt*W.. of plane z
//   B(z, rg)     x-inverse of the six fields on rows rg*G.. of plane z,
//                1/N^2-scaled u x omega, x-forward of the three products
//   C(z, f, xt)  y-forward of product f (0..2) on x columns of plane z
//
// Items are handed out by an atomic ticket in the order
//   segment s: A(s), B(s - D), C(s - 2D)      (s = 0 .. nz + 2D - 1)
// B(z) waits until all A(z) items have signalled, C(z) until all B(z) have.
// A consumer only waits on items with smaller tickets, which were handed to
// CTAs that are already running, so the schedule cannot deadlock; each wait
// is bounded (`spin_limit` polls) and a timeout sets an error word instead of
// hanging.  Reads of data produced inside the launch bypass L1 (ld.global.cg).
// After B has read a plane's omega rows they are discarded from L2
// (discard.global.L2) so the dead data is never written back to HBM.
// HBM traffic of the phase: the six fields read once, three written once.
#include <stdlib.h>

#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_xy.cuh"

namespace sns {

namespace {

enum ItemType : int { ITEM_A = 0, ITEM_B = 1, ITEM_C = 2, ITEM_DONE = 3 };

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void discard_l2_line(const void* p) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

template <typename C>
__device__ __forceinline__ C ldcg(const C* p) {
  return __ldcg(p);
}

// cumulative number of items in segments [0, s)
__device__ __forceinline__ long long items_before(int s, const XYArgs& a) {
  auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
  return (long long)a.nA * clampi(s, 0, a.nz) + (long long)a.nB * clampi(s - a.D, 0, a.nz) +
         (long long)a.nC * clampi(s - 2 * a.D, 0, a.nz);
}

// ticket -> (type, plane, index within the plane)
__device__ void decode(long long t, const XYArgs& a, int* type, int* plane, int* index) {
  const int nseg = a.nz + 2 * a.D;
  if (t >= items_before(nseg, a)) {
    *type = ITEM_DONE;
    return;
  }
  int lo = 0, hi = nseg - 1;  // largest s with items_before(s) <= t
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (items_before(mid, a) <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  const int s = lo;
  long long o = t - items_before(s, a);
  const int na = (s < a.nz) ? a.nA : 0;
  const int nb = (s - a.D >= 0 && s - a.D < a.nz) ? a.nB : 0;
  if (o < na) {
    *type = ITEM_A;
    *plane = s;
    *index = (int)o;
    return;
  }
  o -= na;
  if (o < nb) {
    *type = ITEM_B;
    *plane = s - a.D;
    *index = (int)o;
    return;
  }
  o -= nb;
  *type = ITEM_C;
  *plane = s - 2 * a.D;
  *index = (int)o;
}

// y lines of three fields (U[f0..f0+2]) on W adjacent x columns of plane z,
// in place.  Thread t owns field f0 + t / (W*TPL), x column w = t mod W and
// positions j + e*TPL of that line (j = (t / W) mod TPL): consecutive threads
// read adjacent x, so the loads are coalesced W elements wide.
template <typename T, int LY>
__device__ __forceinline__ void item_ylines(const XYArgs& a, cx_t<T>* sm, int f0, int z, int x0,
                                            const cx_t<T>* tw, T sg) {
  using C = cx_t<T>;
  using P = LinePlan<LY>;
  constexpr int E = P::E, TPL = P::TPL;
  const int W = a.W;
  const int RS = tile_stride(LY, W, (int)sizeof(C));
  const int t = threadIdx.x;
  const int fi = t / (W * TPL), rest = t - fi * (W * TPL);
  const int w = rest % W, j = rest / W;
  C* data = reinterpret_cast<C*>(a.U[f0 + fi]);
  const int64_t nxy = (int64_t)a.nx * a.ny;
  const int64_t i0 = (int64_t)z * nxy + x0 + w + (int64_t)a.nx * j;
  const int64_t step = (int64_t)a.nx * TPL;
  C v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = ldcg(data + i0 + e * step);
  line_fft<LY, true>(v, sm + (fi * W + w) * RS, j, tw, sg);
#pragma unroll
  for (int e = 0; e < E; e++) data[i0 + e * step] = v[e];
}

// x lines of the six fields on G rows of plane z: inverse, cross, forward.
template <typename T, int LX>
__device__ __forceinline__ void item_xcross(const XYArgs& a, cx_t<T>* sm, int z, int rg,
                                            const cx_t<T>* tw) {
  using C = cx_t<T>;
  using P = LinePlan<LX>;
  constexpr int E = P::E, TPL = P::TPL, RS = xrow_stride(LX, (int)sizeof(C));
  const int G = a.G;
  const int t = threadIdx.x;
  const int line = t / TPL, j = t % TPL;
  const int fld = line / G;
  const int gl = line - fld * G;
  C* row = sm + line * RS;
  const int64_t rowidx = (int64_t)z * a.ny + (int64_t)rg * G + gl;  // global row number
  const int64_t i0 = rowidx * LX + j;
  C v[E];
  {
    const C* src = reinterpret_cast<const C*>(a.U[fld]);
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = ldcg(src + i0 + TPL * e);
  }
  line_fft<LX, true>(v, row, j, tw, (T)1);
#pragma unroll
  for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
  __syncthreads();
  // every thread has read its omega rows: drop them from L2 without write-back
  {
    const int lines_per_row = (LX * (int)sizeof(C)) / 128;
    const int nlines = 3 * G * lines_per_row;
    for (int q = t; q < nlines; q += blockDim.x) {
      const int f = q / (G * lines_per_row);
      const int r = (q / lines_per_row) % G;
      const int c = q % lines_per_row;
      const C* base = reinterpret_cast<const C*>(a.U[3 + f]) +
                      ((int64_t)z * a.ny + (int64_t)rg * G + r) * LX;
      discard_l2_line(reinterpret_cast<const char*>(base) + 128 * c);
    }
  }
  const int per = G * LX;
  for (int q = t; q < per; q += blockDim.x) {
    const int g = q / LX, p = q & (LX - 1);
    C u[3], w[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      u[d] = sm[(d * G + g) * RS + pad_pos(p)];
      w[d] = sm[((3 + d) * G + g) * RS + pad_pos(p)];
    }
    const T s2 = (T)a.scale2;
    sm[(0 * G + g) * RS + pad_pos(p)] = cscale(s2, csub(cmul(u[1], w[2]), cmul(u[2], w[1])));
    sm[(1 * G + g) * RS + pad_pos(p)] = cscale(s2, csub(cmul(u[2], w[0]), cmul(u[0], w[2])));
    sm[(2 * G + g) * RS + pad_pos(p)] = cscale(s2, csub(cmul(u[0], w[1]), cmul(u[1], w[0])));
  }
  __syncthreads();
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = row[pad_pos(j + TPL * e)];
  __syncthreads();
  line_fft<LX, true>(v, row, j, tw, (T)-1);
  if (fld < 3) {
    C* dst = reinterpret_cast<C*>(a.U[fld]);
#pragma unroll
    for (int e = 0; e < E; e++) dst[i0 + TPL * e] = v[e];
  }
}

template <typename T, int LX, int LY>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_xy_dataflow(const XYArgs a, const cx_t<T>* __restrict__ twx,
                  const cx_t<T>* __restrict__ twy) {
  using C = cx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  __shared__ int s_item[3];
  const int xtiles = a.nx / a.W;
  for (;;) {
    if (threadIdx.x == 0) {
      const long long t = atomicAdd(a.ticket, 1ull);
      int type = ITEM_DONE, plane = 0, index = 0;
      decode(t, a, &type, &plane, &index);
      // wait for the producers of this plane (bounded)
      if (type == ITEM_B || type == ITEM_C) {
        const int* cnt = (type == ITEM_B) ? a.cntA + plane : a.cntB + plane;
        const int target = (type == ITEM_B) ? a.nA : a.nB;
        long long polls = 0;
        while (ld_acquire(cnt) < target) {
          // give up after the poll budget, or at once when another CTA has
          // already given up, so a broken schedule ends the launch quickly
          if (++polls > a.spin_limit || *(volatile int*)a.err) {
            atomicOr(a.err, 1);
            break;
          }
          __nanosleep(64);
        }
      }
      s_item[0] = type;
      s_item[1] = plane;
      s_item[2] = index;
    }
    __syncthreads();
    const int type = s_item[0], z = s_item[1], idx = s_item[2];
    if (type == ITEM_DONE) break;
    if (type == ITEM_A) {  // fields 0..2 then 3..5
      const int fg = idx / xtiles, xt = idx % xtiles;
      item_ylines<T, LY>(a, sm, 3 * fg, z, xt * a.W, twy, (T)1);
    } else if (type == ITEM_B) {
      item_xcross<T, LX>(a, sm, z, idx, twx);
    } else {
      item_ylines<T, LY>(a, sm, 0, z, idx * a.W, twy, (T)-1);
    }
    // publish: every thread orders its own stores at device scope, the block
    // barrier gathers them, then one thread bumps the plane counter
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0 && type != ITEM_C) atomicAdd(type == ITEM_A ? a.cntA + z : a.cntB + z, 1);
  }
}

template <typename T, int LX, int LY>
int launch_xy(const XYPlan& p, XYArgs a, cudaStream_t s) {
  using C = cx_t<T>;
  static bool attr[64] = {false};
  static int occ[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  const size_t smem = p.smem_bytes;
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_xy_dataflow<T, LX, LY>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_xy_dataflow)");
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_xy_dataflow<T, LX, LY>,
                                                      p.threads, smem);
    if (e != cudaSuccess) return cuda_status(e, "occupancy(k_xy_dataflow)");
    occ[dev & 63] = per_sm < 1 ? 1 : per_sm;
    attr[dev & 63] = true;
  }
  const int prec = sizeof(T) == 8 ? PREC_C128 : PREC_C64;
  const C* twx = reinterpret_cast<const C*>(twiddles(LX, prec));
  const C* twy = reinterpret_cast<const C*>(twiddles(LY, prec));
  if (!twx || !twy) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  const long long total = (long long)(p.nA + p.nB + p.nC) * p.nz;
  long long grid = (long long)occ[dev & 63] * sm_count();
  if (grid > total) grid = total;
  // reset the ticket and the per-plane counters (the error word is kept)
  cudaError_t e = cudaMemsetAsync(p.sync_words, 0, p.sync_bytes_to_clear, s);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(xy counters)");
  k_xy_dataflow<T, LX, LY><<<(unsigned)grid, p.threads, smem, s>>>(a, twx, twy);
  SNS_CHECK_LAUNCH("k_xy_dataflow");
  return OK;
}

int elems_of(int L) { return L >= 16 ? 16 : L; }

}  // namespace

bool xy_supported(int nx, int ny, int prec) {
  (void)prec;
  return nx == ny && (nx == 64 || nx == 128 || nx == 256 || nx == 512);
}

int xy_plan(XYPlan& p, int nx, int ny, int nz, int prec) {
  p = XYPlan{};
  if (!xy_supported(nx, ny, prec)) {
    set_error("xy dataflow pass: unsupported plane size");
    return ERR_UNSUPPORTED;
  }
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  p.prec = prec;
  const size_t esz = prec == PREC_C128 ? 16 : 8;
  const int tplx = nx / elems_of(nx), tply = ny / elems_of(ny);
  // A and C items transform three fields of W adjacent y lines (3*W*tply
  // threads), B items the six fields of G rows (6*G*tplx threads): the two
  // counts match when G = W*tply / (2*tplx).
  int W = prec == PREC_C128 ? 8 : 16;
  // tile width override for tuning sweeps (SNS_XY_W, a power of two)
  if (const char* e = getenv("SNS_XY_W")) {
    const int v = atoi(e);
    if (v >= 1 && (v & (v - 1)) == 0) W = v;
  }
  while (W > 1 && (W > nx || 3 * W * tply > max_threads(prec))) W /= 2;
  const int G = W * tply / (2 * tplx);
  if (G < 1 || ny % G != 0 || 3 * W * tply > max_threads(prec)) {
    set_error("xy dataflow pass: no tile layout for this plane");
    return ERR_UNSUPPORTED;
  }
  p.W = W;
  p.G = G;
  p.threads = 3 * W * tply;
  p.smem_bytes = (size_t)(3 * W) * tile_stride(ny, W, (int)esz) * esz;
  if ((size_t)(6 * G) * xrow_stride(nx, (int)esz) * esz > p.smem_bytes)
    p.smem_bytes = (size_t)(6 * G) * xrow_stride(nx, (int)esz) * esz;
  p.nA = 2 * (nx / W);
  p.nB = ny / G;
  p.nC = nx / W;
  // lag (in planes) between the item kinds: enough that the producers of a
  // plane have finished when its consumers are handed out
  p.D = 4;
  if (const char* e = getenv("SNS_XY_LAG")) {
    const int v = atoi(e);
    if (v >= 1 && v <= 64) p.D = v;
  }
  return OK;
}

int xy_run(const XYPlan& p, void* const U[6], int* sync_words, cudaStream_t s) {
  XYArgs a{};
  for (int i = 0; i < 6; i++) a.U[i] = U[i];
  a.nx = p.nx;
  a.ny = p.ny;
  a.nz = p.nz;
  a.W = p.W;
  a.G = p.G;
  a.nA = p.nA;
  a.nB = p.nB;
  a.nC = p.nC;
  a.D = p.D;
  const double N = (double)p.nx * p.ny * p.nz;
  a.scale2 = 1.0 / (N * N);
  // layout of sync_words: [ticket (2 ints)][cntA nz][cntB nz][err]
  a.ticket = reinterpret_cast<unsigned long long*>(sync_words);
  a.cntA = sync_words + 2;
  a.cntB = sync_words + 2 + p.nz;
  a.err = sync_words + 2 + 2 * p.nz;
  a.spin_limit = 4000000;  // a few hundred ms of 64 ns sleeps; producers take microseconds
  // SNS_XY_SPIN=<polls>: a smaller budget (a test of the timeout path)
  if (const char* e = getenv("SNS_XY_SPIN")) {
    const long long v = atoll(e);
    if (v >= 1 && v < a.spin_limit) a.spin_limit = v;
  }
  XYPlan q = p;
  q.sync_words = sync_words;
  q.sync_bytes_to_clear = sizeof(int) * (2 + 2 * (size_t)p.nz);
  if (p.prec == PREC_C128) {
    switch (p.nx) {
      case 64: return launch_xy<double, 64, 64>(q, a, s);
      case 128: return launch_xy<double, 128, 128>(q, a, s);
      case 256: return launch_xy<double, 256, 256>(q, a, s);
      case 512: return launch_xy<double, 512, 512>(q, a, s);
    }
  } else {
    switch (p.nx) {
      case 64: return launch_xy<float, 64, 64>(q, a, s);
      case 128: return launch_xy<float, 128, 128>(q, a, s);
      case 256: return launch_xy<float, 256, 256>(q, a, s);
      case 512: return launch_xy<float, 512, 512>(q, a, s);
    }
  }
  set_error("xy dataflow pass: unsupported plane size");
  return ERR_UNSUPPORTED;
}

size_t xy_sync_words(int nz) { return 2 + 2 * (size_t)nz + 1; }

}  // namespace sns
