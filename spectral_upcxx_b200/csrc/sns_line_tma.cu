// Plain line passes (y or z lines, PRO_LOAD) over TMA-staged tiles.
//
// The direct-load pass (k_line_pass, sns_fft.cu) starts a tile's HBM reads
// only when its CTA starts, so a CTA's loads and its line FFTs never overlap.
// Here a persistent CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x,
// ...; a tile's input -- one field's W x L (x G) box -- comes into a shared
// memory stage as cp.async.bulk.tensor copies on an mbarrier, issued as soon
// as the previous tile's threads have read the stage (one stage) or one tile
// ahead (two stages), so the copy of the next tile runs under the transforms
// and the stores of the current one.  The arithmetic is k_line_pass's on the
// same values (line_pass_tile_staged), so both give the same bits.
//
// Loads read only this GPU's own fields and never use cluster multicast.
// Every wait on a stage is bounded: a wait that runs out records 1 in the
// caller's error word and the CTA stops after one more bounded wait for its
// copies in flight; a box that fails the kernel's own alignment and range
// check records 2 and is not loaded.
#include <stdlib.h>

#include <algorithm>
#include <mutex>

#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_tiles.cuh"
#include "sns_tma.cuh"

namespace sns {

namespace {

// A field's tensor map, selected with constant indices.
__device__ __forceinline__ const CUtensorMap* pick_map(
    int i, const CUtensorMap& m0, const CUtensorMap& m1, const CUtensorMap& m2,
    const CUtensorMap& m3, const CUtensorMap& m4, const CUtensorMap& m5) {
  return i == 0 ? &m0 : i == 1 ? &m1 : i == 2 ? &m2 : i == 3 ? &m3 : i == 4 ? &m4 : &m5;
}

// The box of one tile: (W, L, G) for y lines (groups along z), (W, G, L) for
// z lines (groups along y); along the line at most 256 positions per box.
constexpr int kMaxTmaFields = 6;

}  // namespace

template <typename T, int L, int ORD, int S>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_line_tma(const __grid_constant__ CUtensorMap m0, const __grid_constant__ CUtensorMap m1,
               const __grid_constant__ CUtensorMap m2, const __grid_constant__ CUtensorMap m3,
               const __grid_constant__ CUtensorMap m4, const __grid_constant__ CUtensorMap m5,
               const LineGeo geo, const FieldPtrs f, const cx_t<T>* __restrict__ tw, T sg,
               T scale, int flags, int wshift, int* err, long long stall_cycles) {
  using C = cx_t<T>;
  constexpr int LB = L < 256 ? L : 256;  // line positions per box
  // the stages start at the first 128-byte boundary of the dynamic block (the
  // launch adds the slack), then the exchange rows, then the mbarriers (the
  // stages', then the stall test's)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = geo.W, G = geo.G, lines = W * G;
  const int per = lines * L;
  const bool ylines = geo.axis == 1, xlines = geo.axis == 0;
  const uint32_t raw = tc::smem_u32(smem_raw);
  C* stage0 = reinterpret_cast<C*>(smem_raw + (((raw + 127u) & ~127u) - raw));
  C* rows = stage0 + S * per;
  uint64_t* full = reinterpret_cast<uint64_t*>(rows + lines * tile_stride(L, W, (int)sizeof(C)));
  const int nf = f.n;
  const int64_t ntiles = geo.TA * geo.TB * nf;
  const int64_t stride = gridDim.x;
  pdl_trigger();
  if (threadIdx.x == 0) {
    for (int k = 0; k <= S; k++) tc::mbar_init(&full[k], 1);
    for (int i = 0; i < nf; i++) tma::prefetch_map(pick_map(i, m0, m1, m2, m3, m4, m5));
  }
  __syncthreads();
  // the fields are written by the pass before
  pdl_wait();
  auto issue = [&](int64_t blk, int k) {  // thread 0
    const int fld = (int)(blk % nf);
    const int64_t t = blk / nf;
    const CUtensorMap* m = pick_map(fld, m0, m1, m2, m3, m4, m5);
    const int u = (int)(sizeof(C) / 8);
    C* st = stage0 + k * per;
    if (xlines) {
      // G whole rows of one xy plane: one (nx, G, 1) box at row r0 = t G
      const int64_t r0 = t * G;
      const int y0 = (int)(r0 % geo.ny), z0 = (int)(r0 / geo.ny);
      if (y0 + G > geo.ny || z0 >= geo.nz || (tc::smem_u32(st) & 127u)) {
        atomicExch(err, 2);
        tma::arrive(&full[k]);
        return;
      }
      tma::expect_tx(&full[k], (uint32_t)(per * sizeof(C)));
      tma::load_3d(st, m, 0, y0, z0, &full[k]);
      return;
    }
    const int x0 = (int)((t % geo.TA) * W) * u;
    const int g0 = (int)((t / geo.TA) * G);
    // self-check of the box (16-byte aligned x, inside the field, 128-byte
    // aligned destination): a bad one is recorded and not loaded, and the
    // stage's barrier is released without it
    if ((x0 & 1) || x0 + W * u > geo.nx * u || g0 + G > (ylines ? geo.nz : geo.ny) ||
        (tc::smem_u32(st) & 127u)) {
      atomicExch(err, 2);
      tma::arrive(&full[k]);
      return;
    }
    tma::expect_tx(&full[k], (uint32_t)(per * sizeof(C)));
#pragma unroll 1
    for (int p0 = 0; p0 < L; p0 += LB) {
      if (ylines)
        tma::load_3d(st + p0 * W, m, x0, p0, g0, &full[k]);
      else
        tma::load_3d(st + p0 * lines, m, x0, g0, p0, &full[k]);
    }
  };
  const int64_t first = blockIdx.x;
  if (threadIdx.x == 0 && first < ntiles) issue(first, 0);
  int it = 0;
#pragma unroll 1
  for (int64_t blk = first; blk < ntiles; blk += stride, it++) {
    const int k = S == 1 ? 0 : (it & 1);
    const uint32_t par = S == 1 ? (uint32_t)(it & 1) : (uint32_t)((it >> 1) & 1);
    const bool more = blk + stride < ntiles;
    if (S == 2 && threadIdx.x == 0 && more) {
      // stage k ^ 1 was last read by the previous tile, before the barrier
      // that closed it
      tma::fence_proxy_async();
      issue(blk + stride, k ^ 1);
    }
    bool ok = tc::mbar_wait(&full[k], par, tc::kWaitCycles);
    if (stall_cycles > 0 && it == 0) ok = ok && tc::mbar_wait(&full[S], 0, stall_cycles);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        tc::mbar_wait(&full[k], par, tc::kWaitCycles);
        if (S == 2 && more)
          tc::mbar_wait(&full[k ^ 1], (uint32_t)(((it + 1) >> 1) & 1), tc::kWaitCycles);
      }
      __syncthreads();
      return;
    }
    line_pass_tile_staged<T, L, ParamFields, ORD>(geo, ParamFields{f}, nf, tw, sg, scale, flags,
                                                  wshift, blk, stage0 + k * per, rows, [&] {
                                                    if (S == 1) {
                                                      __syncthreads();
                                                      if (threadIdx.x == 0 && more) {
                                                        tma::fence_proxy_async();
                                                        issue(blk + stride, 0);
                                                      }
                                                    }
                                                  });
    // the stage and the rows are free for the next tile
    __syncthreads();
  }
}

namespace {

// Stall test of the TMA-staged passes (SNS_TMA_STALL_TEST=<cycles>; 0: none).
long long line_tma_stall_cycles() {
  const char* e = getenv("SNS_TMA_STALL_TEST");
  const long long v = e ? atoll(e) : 0;
  return v > 0 ? v : 0;
}

size_t line_tma_smem(int L, int W, int G, int S, size_t esz) {
  return ((size_t)S * W * G * L + (size_t)W * G * tile_stride(L, W, (int)esz)) * esz + 128 +
         8 * (S + 1);
}

template <typename T, int L, int ORD, int S>
int launch_line_tma(const LineGeo& geo, const FieldPtrs& f, int sign, int flags, double scale,
                    cudaStream_t s, int* err) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  constexpr int LB = L < 256 ? L : 256;
  const int esz = (int)sizeof(C);
  const bool ylines = geo.axis == 1;
  const int threads = geo.W * geo.G * TPL;
  const size_t smem = line_tma_smem(L, geo.W, geo.G, S, sizeof(C));
  CUtensorMap m[kMaxTmaFields];
  for (int i = 0; i < f.n; i++) {
    const int rc = geo.axis == 0
                       ? field_tensor_map(&m[i], f.in[i], geo.nx, geo.ny, geo.nz, esz, geo.nx,
                                          geo.G, 1)
                   : ylines ? field_tensor_map(&m[i], f.in[i], geo.nx, geo.ny, geo.nz, esz,
                                               geo.W, LB, geo.G)
                            : field_tensor_map(&m[i], f.in[i], geo.nx, geo.ny, geo.nz, esz,
                                               geo.W, geo.G, LB);
    if (rc) return rc;
  }
  for (int i = f.n; i < kMaxTmaFields; i++) m[i] = m[0];
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_line_tma<T, L, ORD, S>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_line_tma)");
    attr[dev & 63] = true;
  }
  int per_sm = 0;
  cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_line_tma<T, L, ORD, S>, threads, smem);
  if (e != cudaSuccess) return cuda_status(e, "occupancy(k_line_tma)");
  if (per_sm < 1) {
    set_error("TMA-staged line pass: the tile does not fit on an SM");
    return ERR_UNSUPPORTED;
  }
  const int64_t ntiles = geo.TA * geo.TB * f.n;
  const int blocks = (int)std::min<int64_t>(ntiles, (int64_t)per_sm * sm_count());
  const C* tw = reinterpret_cast<const C*>(
      geo.tw ? geo.tw : twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  int wshift = 0;
  while ((1 << wshift) < geo.W) wshift++;
  e = launch_pdl(k_line_tma<T, L, ORD, S>, dim3((unsigned)blocks), dim3(threads), smem, s, m[0],
                 m[1], m[2], m[3], m[4], m[5], geo, f, tw, (T)sign, (T)scale, flags, wshift, err,
                 line_tma_stall_cycles());
  if (e != cudaSuccess) return cuda_status(e, "k_line_tma");
  return OK;
}

template <typename T, int L>
int dispatch_line_tma(const LineGeo& geo, const FieldPtrs& f, int sign, int flags, double scale,
                      cudaStream_t s, int stages, int* err) {
  const bool rem = geo.ord == RADIX_REM_FIRST;
  if (stages == 2)
    return rem ? launch_line_tma<T, L, RADIX_REM_FIRST, 2>(geo, f, sign, flags, scale, s, err)
               : launch_line_tma<T, L, RADIX16_FIRST, 2>(geo, f, sign, flags, scale, s, err);
  return rem ? launch_line_tma<T, L, RADIX_REM_FIRST, 1>(geo, f, sign, flags, scale, s, err)
             : launch_line_tma<T, L, RADIX16_FIRST, 1>(geo, f, sign, flags, scale, s, err);
}

}  // namespace

bool line_tma_ok(const LineGeo& geo, int prec, int stages) {
  const int L = geo.L;
  if (geo.axis != 0 && geo.axis != 1 && geo.axis != 2) return false;
  if (L != 32 && L != 64 && L != 128 && L != 256 && L != 512) return false;
  if (geo.ord != RADIX16_FIRST && geo.ord != RADIX_REM_FIRST) return false;
  if (stages != 1 && stages != 2) return false;
  const int esz = prec == PREC_C128 ? 16 : 8;
  const int LB = L < 256 ? L : 256;
  const bool ylines = geo.axis == 1;
  // y-line boxes of more than 256 positions are split along y, which keeps
  // the stage in [z][y][x] order only for one group
  if (ylines && L > 256 && geo.G != 1) return false;
  const int TPL = L / 16;
  if (geo.W * geo.G * TPL > max_threads(prec)) return false;
  if (line_tma_smem(L, geo.W, geo.G, stages, esz) > 220 * 1024) return false;
  // x lines: G whole rows of one plane per box, at most 256 units (8 bytes) long
  if (geo.axis == 0)
    return geo.W == 1 && geo.ny % geo.G == 0 && field_box_ok(geo.nx, geo.ny, geo.nz, esz, geo.nx,
                                                              geo.G, 1);
  return ylines ? field_box_ok(geo.nx, geo.ny, geo.nz, esz, geo.W, LB, geo.G)
                : field_box_ok(geo.nx, geo.ny, geo.nz, esz, geo.W, geo.G, LB);
}

int run_line_pass_tma(const LineGeo& geo, const FieldPtrs& f, int sign, int flags, double scale,
                      int prec, cudaStream_t s, int stages, int* err) {
  if (f.n < 1 || f.n > kMaxTmaFields || !err) {
    set_error("TMA-staged line pass: 1..6 fields and an error word");
    return ERR_ARG;
  }
  if (!line_tma_ok(geo, prec, stages)) {
    set_error("TMA-staged line pass: the tile is not loadable by the TMA");
    return ERR_UNSUPPORTED;
  }
  for (int i = 0; i < f.n; i++)
    if (!f.in[i] || !f.out[i]) {
      set_error("TMA-staged line pass: null field");
      return ERR_ARG;
    }
  const bool d = prec == PREC_C128;
  switch (geo.L) {
#define SNS_LINE_TMA_CASE(L)                                                                   \
  case L:                                                                                      \
    return d ? dispatch_line_tma<double, L>(geo, f, sign, flags, scale, s, stages, err)        \
             : dispatch_line_tma<float, L>(geo, f, sign, flags, scale, s, stages, err);
    SNS_LINE_TMA_CASE(32)
    SNS_LINE_TMA_CASE(64)
    SNS_LINE_TMA_CASE(128)
    SNS_LINE_TMA_CASE(256)
    SNS_LINE_TMA_CASE(512)
#undef SNS_LINE_TMA_CASE
    default:
      set_error("TMA-staged line pass: line length not supported");
      return ERR_UNSUPPORTED;
  }
}

}  // namespace sns

namespace sns {

// Error word of the 3D transform's TMA-staged passes (they have no stepper
// whose word they could use): one per device that loads the library.
static __device__ int g_fft_tma_err;

int* fft_tma_err_word() {
  static std::mutex mu;
  static int* addr[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_fft_tma_err) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    addr[dev] = static_cast<int*>(p);
  }
  return addr[dev];
}

int fft_tma_check(cudaStream_t s) {
  int* w = fft_tma_err_word();
  if (!w) return OK;  // no word: no TMA-staged pass ran on this device
  int err = 0;
  int rc = cuda_status(cudaMemcpyAsync(&err, w, sizeof(int), cudaMemcpyDeviceToHost, s),
                       "sns_fft_check");
  if (rc) return rc;
  if ((rc = cuda_status(cudaStreamSynchronize(s), "sns_fft_check"))) return rc;
  if (err) {
    cudaMemsetAsync(w, 0, sizeof(int), s);
    cudaStreamSynchronize(s);
    set_error(err == 2 ? "3D transform: a TMA-staged pass refused a tile box (alignment or "
                         "range); results are invalid"
                       : "3D transform: a bounded wait of a TMA-staged pass gave up; results "
                         "are invalid");
    return ERR_TIMEOUT;
  }
  return OK;
}

}  // namespace sns
