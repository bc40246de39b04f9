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
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <vector>

#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_ns.cuh"
#include "sns_ops.cuh"
#include "sns_tiles.cuh"
#include "sns_tma.cuh"

namespace sns {

// ---------------------------------------------------------------------------
// K3: x lines -- inverse 6 fields, cross product, forward 3 fields.
template <typename T, int L>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_xcross(FieldPtrs f, const cx_t<T>* __restrict__ tw, int G, T scale2, int64_t pf) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_trigger();
  pdl_wait();
  xcross_tile<T, L>(ParamFields{f}, tw, G, scale2, (int64_t)blockIdx.x, (int)blockDim.x,
                    reinterpret_cast<cx_t<T>*>(smem_raw), pf, (int64_t)gridDim.x);
}

// K3 for CTAs of at most 192 threads, compiled for five resident CTAs per SM
// (64 registers per thread instead of 80): more warps to hide the row loads'
// latency, at the price of a few spilled registers.
template <typename T, int L>
__global__ void __launch_bounds__(192, 5)
    k_xcross_occ(FieldPtrs f, const cx_t<T>* __restrict__ tw, int G, T scale2, int64_t pf) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_trigger();
  pdl_wait();
  xcross_tile<T, L>(ParamFields{f}, tw, G, scale2, (int64_t)blockIdx.x, (int)blockDim.x,
                    reinterpret_cast<cx_t<T>*>(smem_raw), pf, (int64_t)gridDim.x);
}

// K3 with TMA-staged tiles: a persistent CTA walks the tiles blockIdx.x,
// + gridDim.x, ...; the G rows of each of the six fields of its next tile (G L
// contiguous elements per field) come into a shared-memory stage as six bulk
// copies on an mbarrier, issued as soon as the current tile's threads have
// read the stage into registers, so the loads overlap the transforms and the
// cross product.  Bounded waits and the stall test as in k_zcurl_tma.
template <typename T, int L>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_xcross_tma(FieldPtrs f, const cx_t<T>* __restrict__ tw, int G, T scale2, int64_t ntiles,
                 int* err, long long stall_cycles) {
  using C = cx_t<T>;
  constexpr int E = LinePlan<L>::E, TPL = LinePlan<L>::TPL;
  constexpr int RS = xrow_stride(L, (int)sizeof(C));
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int per = G * L;  // elements of one field's rows of a tile
  const uint32_t raw = tc::smem_u32(smem_raw);
  C* stage = reinterpret_cast<C*>(smem_raw + (((raw + 127u) & ~127u) - raw));
  C* rows = stage + 6 * per;
  uint64_t* full = reinterpret_cast<uint64_t*>(rows + 6 * G * RS);  // stage, stall test
  const int64_t stride = gridDim.x;
  pdl_trigger();
  if (threadIdx.x == 0) {
    tc::mbar_init(&full[0], 1);
    tc::mbar_init(&full[1], 1);
  }
  __syncthreads();
  pdl_wait();  // the rows are written by the y pass before
  auto issue = [&](int64_t blk) {  // thread 0
    const int64_t e0 = blk * per;
    if ((tc::smem_u32(stage) & 127u) || ((e0 * (int64_t)sizeof(C)) & 15)) {
      atomicExch(err, 2);
      tma::arrive(&full[0]);
      return;
    }
    tma::expect_tx(&full[0], (uint32_t)(6 * per * sizeof(C)));
#pragma unroll 1
    for (int fl = 0; fl < 6; fl++)
      tma::load_bulk(stage + fl * per, reinterpret_cast<const C*>(select_ptr(f.in, fl)) + e0,
                     (uint32_t)(per * sizeof(C)), &full[0]);
  };
  if (threadIdx.x == 0 && (int64_t)blockIdx.x < ntiles) issue(blockIdx.x);
  int it = 0;
#pragma unroll 1
  for (int64_t blk = blockIdx.x; blk < ntiles; blk += stride, it++) {
    const bool more = blk + stride < ntiles;
    bool ok = tc::mbar_wait(&full[0], (uint32_t)(it & 1), tc::kWaitCycles);
    if (stall_cycles > 0 && it == 0) ok = ok && tc::mbar_wait(&full[1], 0, stall_cycles);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        tc::mbar_wait(&full[0], (uint32_t)(it & 1), tc::kWaitCycles);
      }
      __syncthreads();
      return;
    }
    xcross_tile_from<T, L>(ParamFields{f}, tw, G, scale2, blk, (int)blockDim.x, rows,
                           [&](int fld, int gl, int j, C (&v)[E]) {
                             const C* src = stage + fld * per + gl * L + j;
#pragma unroll
                             for (int e = 0; e < E; e++) v[e] = src[TPL * e];
                             // every thread has read the stage: refill it
                             __syncthreads();
                             if (threadIdx.x == 0 && more) {
                               tma::fence_proxy_async();
                               issue(blk + stride);
                             }
                           });
    // the rows are free for the next tile
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// K3 of a real-field run: rows of the half spectrum, M = nx/2 values
// (kx = 0 .. M-1; kx = M is a Nyquist mode, zero).  Inverse: the real line u of
// length 2M comes from one M-point complex FFT of
//   Z[k] = (V[k] + conj V[M-k]) + i w^k (V[k] - conj V[M-k]),  w = e^{+2 pi i/2M},
// V[M] = 0, as z[m] = u[2m] + i u[2m+1].  The cross product acts on the two real
// samples of every complex slot.  Forward: Z = FFT_M(c[2m] + i c[2m+1]) and
//   C[k] = (Z[k] + conj Z[M-k]) / 2 - i W^k (Z[k] - conj Z[M-k]) / 2,  W = e^{-2 pi i/2M}.
// twN: the 2M-point table exp(-2 pi i m / 2M); twM: the M-point table.
// The pre- and post-processing run on pairs (k, M-k) in shared memory, so no
// line values stay in registers across them; FP32 fits two CTAs per SM.
template <typename T, int M>
__global__ void __launch_bounds__(384, sizeof(T) == 4 ? 2 : 1)
    k_xcross_r2c(FieldPtrs f, const cx_t<T>* __restrict__ twN, const cx_t<T>* __restrict__ twM,
                 int G, T scale2) {
  using C = cx_t<T>;
  using P = LinePlan<M>;
  constexpr int E = P::E, TPL = P::TPL, RS = xrow_stride(M, (int)sizeof(C));
  static_assert(TPL <= 32, "a line's threads share a warp");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_trigger();
  pdl_wait();
  C* sm = reinterpret_cast<C*>(smem_raw);
  const int64_t row0 = (int64_t)blockIdx.x * G;
  const int per = G * M;
  const int j = threadIdx.x % TPL, line = threadIdx.x / TPL;
  const int fld = line / G, gl = line - fld * G;
  C* row = sm + line * RS;
  C v[E];
  {
    const C* __restrict__ src = reinterpret_cast<const C*>(select_ptr(f.in, fld));
    const int64_t i0 = (row0 + gl) * M + j;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[i0 + TPL * e];
  }
#pragma unroll
  for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
  line_sync<TPL>();
  // Z in place, one thread per pair (k, M-k):  with A = V[k] + conj V[M-k] and
  // B = V[k] - conj V[M-k],  Z[k] = A + i w^k B  and  Z[M-k] = conj(A - i w^k B)
#pragma unroll 1
  for (int e = 0; e <= M / (2 * TPL); e++) {
    const int k = j + TPL * e;
    if (k <= M / 2) {
      const C vk = row[pad_pos(k)];
      const C vm = k == 0 ? mk((T)0, (T)0) : row[pad_pos(M - k)];
      const C vmc = mk(vm.x, -vm.y);
      const C a = cadd(vk, vmc), b = csub(vk, vmc);
      const C wb = cmul(mk(twN[k].x, -twN[k].y), b);  // w^k b, w = e^{+2 pi i / 2M}
      row[pad_pos(k)] = mk(a.x - wb.y, a.y + wb.x);
      if (k > 0 && k < M / 2) row[pad_pos(M - k)] = mk(a.x + wb.y, wb.x - a.y);
    }
  }
  line_sync<TPL>();
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = row[pad_pos(j + TPL * e)];
  line_sync<TPL>();
  line_fft<M>(v, row, j, twM, (T)1);
#pragma unroll
  for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
  __syncthreads();

  // c = (u/N) x (omega/N) on the real samples (.x and .y of each slot)
  for (int q = threadIdx.x; q < per; q += blockDim.x) {
    const int g = q / M, p = q & (M - 1);
    C u[3], w[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      u[d] = sm[(d * G + g) * RS + pad_pos(p)];
      w[d] = sm[((3 + d) * G + g) * RS + pad_pos(p)];
    }
    const C c0 = mk(u[1].x * w[2].x - u[2].x * w[1].x, u[1].y * w[2].y - u[2].y * w[1].y);
    const C c1 = mk(u[2].x * w[0].x - u[0].x * w[2].x, u[2].y * w[0].y - u[0].y * w[2].y);
    const C c2 = mk(u[0].x * w[1].x - u[1].x * w[0].x, u[0].y * w[1].y - u[1].y * w[0].y);
    sm[(0 * G + g) * RS + pad_pos(p)] = cscale(scale2, c0);
    sm[(1 * G + g) * RS + pad_pos(p)] = cscale(scale2, c1);
    sm[(2 * G + g) * RS + pad_pos(p)] = cscale(scale2, c2);
  }
  __syncthreads();

  // forward: warps holding only omega rows skip it (as in k_xcross)
  constexpr int kLinesPerWarp = 32 / TPL;
  const bool skip = (G % kLinesPerWarp == 0) && fld >= 3;
  if (!skip) {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = row[pad_pos(j + TPL * e)];
    line_sync<TPL>();
    line_fft<M>(v, row, j, twM, (T)-1);
#pragma unroll
    for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
    line_sync<TPL>();
  }
  if (fld < 3) {
    // one thread per pair (k, M-k):  with Ev = (Z[k] + conj Z[M-k]) / 2 and
    // Od = (Z[k] - conj Z[M-k]) / 2,  C[k] = Ev - i W^k Od  and
    // C[M-k] = conj(Ev + i W^k Od)
    C* __restrict__ dst = reinterpret_cast<C*>(select_ptr(f.out, fld)) + (row0 + gl) * M;
#pragma unroll 1
    for (int e = 0; e <= M / (2 * TPL); e++) {
      const int k = j + TPL * e;
      if (k <= M / 2) {
        const C z = row[pad_pos(k)];
        const C zm = row[pad_pos(k == 0 ? 0 : M - k)];
        const C ev = mk((T)0.5 * (z.x + zm.x), (T)0.5 * (z.y - zm.y));
        const C od = mk((T)0.5 * (z.x - zm.x), (T)0.5 * (z.y + zm.y));
        const C wo = cmul(twN[k], od);  // W^k od
        dst[k] = mk(ev.x + wo.y, ev.y - wo.x);
        if (k > 0 && k < M / 2) dst[M - k] = mk(ev.x - wo.y, -(ev.y + wo.x));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// K1: z lines -- inverse of V and of omega = i k x V from one load of V.
template <typename T, int L, bool RELOAD>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_zcurl(const LineGeo geo, const FieldPtrs f, const cx_t<T>* __restrict__ tw, int wshift) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_trigger();
  pdl_wait();
  if constexpr (RELOAD)
    curl_zpass_tile_reload<T, L>(geo, ParamFields{f}, tw, wshift, (int64_t)blockIdx.x,
                                 reinterpret_cast<cx_t<T>*>(smem_raw));
  else
    curl_zpass_tile<T, L>(geo, ParamFields{f}, tw, wshift, (int64_t)blockIdx.x,
                          reinterpret_cast<cx_t<T>*>(smem_raw));
}

// K1 with TMA-staged tiles.  A persistent CTA walks the tiles blockIdx.x,
// blockIdx.x + gridDim.x, ...; the three components of V of a tile come into
// shared memory as TMA boxes (W x G x L elements each, one box per component
// and 256 z planes) while the CTA transforms the tile before it, so the
// HBM reads overlap the line FFTs instead of preceding them.  S = 2: two
// stages, the next tile's load is issued as the current tile starts; S = 1:
// one stage, refilled as soon as the current tile's last read of it is done
// (before its omega transforms).  Every wait on a stage is bounded: a wait
// that runs out sets *err, waits (with the full budget again) for the CTA's
// copies still in flight and ends the CTA.  stall_cycles > 0 is the test of
// that path: the first tile's wait also waits that long on a barrier that
// nothing arrives at.
template <typename T, int L, int S>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_zcurl_tma(const __grid_constant__ CUtensorMap m0, const __grid_constant__ CUtensorMap m1,
                const __grid_constant__ CUtensorMap m2, const LineGeo geo, const FieldPtrs f,
                const cx_t<T>* __restrict__ tw, int wshift, int* err, long long stall_cycles) {
  using C = cx_t<T>;
  constexpr int ZB = L < 256 ? L : 256;  // z planes per box
  // the TMA writes to 128-byte aligned shared memory: the stages start at the
  // first 128-byte boundary of the dynamic block (the launch adds the slack),
  // then the rows, then the mbarriers (the stages', then the stall test's)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lines = geo.W * geo.G;
  const int comp = lines * L;  // elements of one component's tile
  const uint32_t raw = tc::smem_u32(smem_raw);
  C* stage0 = reinterpret_cast<C*>(smem_raw + (((raw + 127u) & ~127u) - raw));
  C* rows = stage0 + S * 3 * comp;
  uint64_t* full = reinterpret_cast<uint64_t*>(rows + 3 * lines * tile_stride(L, geo.W, (int)sizeof(C)));
  const int64_t ntiles = geo.TA * geo.TB;
  const int64_t stride = gridDim.x;
  pdl_trigger();
  if (threadIdx.x == 0) {
    for (int k = 0; k <= S; k++) tc::mbar_init(&full[k], 1);
    tma::prefetch_map(&m0);
    tma::prefetch_map(&m1);
    tma::prefetch_map(&m2);
  }
  __syncthreads();
  // V is written by the step before (its update pass)
  pdl_wait();
  auto issue = [&](int64_t blk, int k) {  // thread 0
    const int u = (int)(sizeof(C) / 8);
    const int x0 = (int)((blk % geo.TA) * geo.W) * u, y0 = (int)((blk / geo.TA) * geo.G);
    C* st = stage0 + k * 3 * comp;
    // self-check of the box (16-byte aligned x, inside the field, 128-byte
    // aligned destination): a bad one is recorded and not loaded, and the
    // stage's barrier is released without it
    if ((x0 & 1) || x0 + geo.W * u > geo.nx * u || y0 + geo.G > geo.ny ||
        (tc::smem_u32(st) & 127u)) {
      atomicExch(err, 2);
      tma::arrive(&full[k]);
      return;
    }
    tma::expect_tx(&full[k], (uint32_t)(3 * comp * sizeof(C)));
#pragma unroll 1
    for (int z0 = 0; z0 < L; z0 += ZB) {
      tma::load_3d(st + z0 * lines, &m0, x0, y0, z0, &full[k]);
      tma::load_3d(st + comp + z0 * lines, &m1, x0, y0, z0, &full[k]);
      tma::load_3d(st + 2 * comp + z0 * lines, &m2, x0, y0, z0, &full[k]);
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
        if (S == 2 && more) tc::mbar_wait(&full[k ^ 1], (uint32_t)(((it + 1) >> 1) & 1), tc::kWaitCycles);
      }
      __syncthreads();
      return;
    }
    curl_zpass_tile_staged<T, L>(geo, ParamFields{f}, tw, wshift, blk, stage0 + k * 3 * comp, rows,
                                 [&] {
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

// ---------------------------------------------------------------------------
// K5: z lines -- forward 3 fields + Nyquist zeroing, then the AB2 /
// projection / CN update per mode.
template <typename T, int L, bool SGS>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_zfwd_update(const UpdateArgs a, const cx_t<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[4][32];
  pdl_trigger();
  pdl_wait();
  zfwd_update_tile<T, L, SGS>(a, tw, (int64_t)blockIdx.x, (int)blockDim.x,
                              reinterpret_cast<cx_t<T>*>(smem_raw), red);
}

// K5 with the next step's K1 carried in it (zfwd_update_curl_tile): the
// update, then the z-inverse of the new V and of i k x V into a.Uo.
template <typename T, int L, bool RELOAD>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_zfwd_update_curl(const UpdateArgs a, const cx_t<T>* __restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[4][32];
  pdl_trigger();
  pdl_wait();
  zfwd_update_curl_tile<T, L, RELOAD>(a, tw, (int64_t)blockIdx.x, (int)blockDim.x,
                                      reinterpret_cast<cx_t<T>*>(smem_raw), red);
}

// K5 with TMA-staged tiles (plain step, no closure).  A persistent CTA walks
// the tiles blockIdx.x, + gridDim.x, ...; the three components of the cross
// product for a tile (W x L boxes) come into a shared-memory stage by TMA, and
// the next tile's boxes are issued as soon as the current tile's threads have
// read the stage into registers, so they load under the current tile's
// transforms and update.  V and C0 are read in the update as before.  The
// diagnostics of each tile go to its own slot of a.stats, as in k_zfwd_update.
// Bounded waits and the stall test as in k_zcurl_tma.
template <typename T, int L>
__global__ void __launch_bounds__(MaxThreads<T>::value)
    k_zfwd_update_tma(const __grid_constant__ CUtensorMap m0, const __grid_constant__ CUtensorMap m1,
                      const __grid_constant__ CUtensorMap m2, const UpdateArgs a,
                      const cx_t<T>* __restrict__ tw, int64_t ntiles, int* err,
                      long long stall_cycles) {
  using C = cx_t<T>;
  constexpr int E = LinePlan<L>::E, TPL = LinePlan<L>::TPL;
  constexpr int ZB = L < 256 ? L : 256;  // z planes per box
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[4][32];
  const int W = a.W;
  const int comp = W * L;  // elements of one component's tile
  const uint32_t raw = tc::smem_u32(smem_raw);
  C* stage = reinterpret_cast<C*>(smem_raw + (((raw + 127u) & ~127u) - raw));
  C* rows = stage + 3 * comp;
  uint64_t* full =
      reinterpret_cast<uint64_t*>(rows + 3 * W * tile_stride(L, W, (int)sizeof(C)));
  const int64_t stride = gridDim.x;
  pdl_trigger();
  if (threadIdx.x == 0) {
    tc::mbar_init(&full[0], 1);
    tc::mbar_init(&full[1], 1);
    tma::prefetch_map(&m0);
    tma::prefetch_map(&m1);
    tma::prefetch_map(&m2);
  }
  __syncthreads();
  pdl_wait();  // the cross product comes from the y pass before
  auto issue = [&](int64_t blk) {  // thread 0
    const int u = (int)(sizeof(C) / 8);
    const int64_t base = blk * W;
    const int x0 = (int)(base & (a.nx - 1)) * u, y0 = (int)(base >> a.lx);
    if ((x0 & 1) || x0 + W * u > a.nx * u || y0 >= a.ny || (tc::smem_u32(stage) & 127u)) {
      atomicExch(err, 2);
      tma::arrive(&full[0]);
      return;
    }
    tma::expect_tx(&full[0], (uint32_t)(3 * comp * sizeof(C)));
#pragma unroll 1
    for (int z0 = 0; z0 < L; z0 += ZB) {
      tma::load_3d(stage + z0 * W, &m0, x0, y0, z0, &full[0]);
      tma::load_3d(stage + comp + z0 * W, &m1, x0, y0, z0, &full[0]);
      tma::load_3d(stage + 2 * comp + z0 * W, &m2, x0, y0, z0, &full[0]);
    }
  };
  if (threadIdx.x == 0 && (int64_t)blockIdx.x < ntiles) issue(blockIdx.x);
  int it = 0;
#pragma unroll 1
  for (int64_t blk = blockIdx.x; blk < ntiles; blk += stride, it++) {
    const bool more = blk + stride < ntiles;
    bool ok = tc::mbar_wait(&full[0], (uint32_t)(it & 1), tc::kWaitCycles);
    if (stall_cycles > 0 && it == 0) ok = ok && tc::mbar_wait(&full[1], 0, stall_cycles);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(err, 1);
        tc::mbar_wait(&full[0], (uint32_t)(it & 1), tc::kWaitCycles);
      }
      __syncthreads();
      return;
    }
    zfwd_update_tile_from<T, L, false>(a, tw, blk, (int)blockDim.x, rows, red,
                                       [&](int fld, int w, int j, C (&v)[E]) {
                                         const C* src = stage + fld * comp + j * W + w;
#pragma unroll
                                         for (int e = 0; e < E; e++) v[e] = src[TPL * e * W];
                                         // every thread has read the stage: refill it
                                         __syncthreads();
                                         if (threadIdx.x == 0 && more) {
                                           tma::fence_proxy_async();
                                           issue(blk + stride);
                                         }
                                       });
    // the rows and the reduction slots are free for the next tile
    __syncthreads();
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
  const size_t smem = (size_t)6 * G * xrow_stride(L, (int)sizeof(C)) * sizeof(C);
  if (pl.x_occ && threads <= 192) {
    static bool attr_o[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr_o[dev & 63]) {
      cudaError_t e = allow_max_dynamic_smem(k_xcross_occ<T, L>);
      if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_xcross_occ)");
      attr_o[dev & 63] = true;
    }
    const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
    const double N = (double)pl.nx * pl.ny * pl.nz;
    const int64_t pf = tiles_in_waves(k_xcross_occ<T, L>, threads, smem, pl.pf_waves);
    cudaError_t e = launch_pdl(k_xcross_occ<T, L>, dim3((unsigned)(rows / G)), dim3(threads), smem,
                               s, f, tw, G, (T)(1.0 / (N * N)), pf);
    if (e != cudaSuccess) return cuda_status(e, "k_xcross_occ");
    return OK;
  }
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
  const int64_t pf = tiles_in_waves(k_xcross<T, L>, threads, smem, pl.pf_waves);
  cudaError_t e = launch_pdl(k_xcross<T, L>, dim3(blocks), dim3(threads), smem, s, f, tw, G,
                             (T)(1.0 / (N * N)), pf);
  if (e != cudaSuccess) return cuda_status(e, "k_xcross");
  return OK;
}

// Stall test of the TMA-staged passes (SNS_TMA_STALL_TEST=<cycles>; 0: none).
inline long long tma_stall_cycles() {
  const char* e = getenv("SNS_TMA_STALL_TEST");
  const long long v = e ? atoll(e) : 0;
  return v > 0 ? v : 0;
}

// Shared memory of the TMA-staged K3: the stage (6 G rows), 128 bytes of
// alignment slack, the 6 G padded rows of the exchanges and two mbarriers.
inline size_t xcross_tma_smem(int L, int G, size_t esz) {
  return ((size_t)6 * G * L + (size_t)6 * G * xrow_stride(L, (int)esz)) * esz + 128 + 16;
}

// Whether the TMA-staged K3 can run G rows per tile on the (complex) box.
bool x_tma_ok(const NSPlan& p, int G) {
  const int TPL = p.nx >= 16 ? p.nx / 16 : 1;
  const size_t esz = p.prec == PREC_C128 ? 16 : 8;
  return !p.real && ((int64_t)p.ny * p.nz) % G == 0 && 6 * G * TPL <= max_threads(p.prec) &&
         xcross_tma_smem(p.nx, G, esz) <= 220 * 1024 && ((size_t)G * p.nx * esz) % 16 == 0;
}

template <typename T, int L>
int launch_xcross_tma(const NSPlan& pl, const FieldPtrs& f, int64_t rows, int* err,
                      cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  const int G = pl.xG;
  const int threads = 6 * G * TPL;
  const size_t smem = xcross_tma_smem(L, G, sizeof(C));
  for (int i = 0; i < 6; i++)
    if (reinterpret_cast<uintptr_t>(f.in[i]) & 15) {
      set_error("K3 TMA tile: a field is not 16-byte aligned");
      return ERR_UNSUPPORTED;
    }
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_xcross_tma<T, L>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_xcross_tma)");
    attr[dev & 63] = true;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_xcross_tma<T, L>,
                                                                threads, smem);
  if (e != cudaSuccess) return cuda_status(e, "occupancy(k_xcross_tma)");
  if (per_sm < 1) {
    set_error("K3 TMA tile: does not fit on an SM");
    return ERR_UNSUPPORTED;
  }
  const int64_t ntiles = rows / G;
  const int blocks = (int)std::min<int64_t>(ntiles, (int64_t)per_sm * sm_count());
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  const double N = (double)pl.nx * pl.ny * pl.nz;
  e = launch_pdl(k_xcross_tma<T, L>, dim3((unsigned)blocks), dim3(threads), smem, s, f, tw, G,
                 (T)(1.0 / (N * N)), ntiles, err, tma_stall_cycles());
  if (e != cudaSuccess) return cuda_status(e, "k_xcross_tma");
  return OK;
}

template <typename T, int L, bool RELOAD>
int launch_zcurl_as(const NSPlan& pl, const FieldPtrs& f, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  LineGeo g{};
  g.L = L;
  g.W = pl.k1W;
  g.G = pl.k1G;
  g.axis = 2;
  g.nx = pl.nx;
  g.ny = pl.ny;
  g.nz = pl.nz;
  g.kx_half = pl.real;
  g.ps = (int64_t)pl.nx * pl.ny;
  g.gs = pl.nx;
  g.TA = pl.nx / g.W;
  g.TB = pl.ny / g.G;
  g.sa = g.W;
  g.sb = (int64_t)g.G * pl.nx;
  const int threads = 3 * g.W * g.G * TPL;
  const size_t smem =
      (size_t)(RELOAD ? 3 : 6) * g.W * g.G * tile_stride(L, g.W, (int)sizeof(C)) * sizeof(C);
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_zcurl<T, L, RELOAD>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_zcurl)");
    attr[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  int wshift = 0;
  while ((1 << wshift) < g.W) wshift++;
  g.pf = tiles_in_waves(k_zcurl<T, L, RELOAD>, threads, smem, pl.pf_waves);
  cudaError_t e = launch_pdl(k_zcurl<T, L, RELOAD>, dim3((unsigned)(g.TA * g.TB)), dim3(threads),
                             smem, s, g, f, tw, wshift);
  if (e != cudaSuccess) return cuda_status(e, "k_zcurl");
  return OK;
}

// Shared memory of the TMA-staged K1: S stages of the three components'
// W x G x L tiles, then the 3 W G padded rows of the line FFTs' exchanges,
// 128 bytes of alignment slack and the S + 1 mbarriers.
inline size_t zcurl_tma_smem(int L, int W, int G, int S, size_t esz) {
  return ((size_t)S * 3 * W * G * L + (size_t)3 * W * G * tile_stride(L, W, (int)esz)) * esz +
         128 + 8 * (size_t)(S + 1);
}

// Whether the TMA-staged K1 can run W x G tiles with S stages on the box.
bool k1_tma_ok(const NSPlan& p, int W, int G, int S) {
  if (p.nz < 16 || p.nz > 1024) return false;
  const int TPL = p.nz / 16;
  const int esz = p.prec == PREC_C128 ? 16 : 8;
  const int zb = p.nz < 256 ? p.nz : 256;
  return p.nx % W == 0 && p.ny % G == 0 && 3 * W * G * TPL <= max_threads(p.prec) &&
         zcurl_tma_smem(p.nz, W, G, S, esz) <= 220 * 1024 &&
         field_box_ok(p.nx, p.ny, p.nz, esz, W, G, zb);
}


template <typename T, int L, int S>
int launch_zcurl_tma(const NSPlan& pl, const FieldPtrs& f, int* err, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  constexpr int ZB = L < 256 ? L : 256;
  LineGeo g{};
  g.L = L;
  g.W = pl.k1W;
  g.G = pl.k1G;
  g.axis = 2;
  g.nx = pl.nx;
  g.ny = pl.ny;
  g.nz = pl.nz;
  g.kx_half = pl.real;
  g.ps = (int64_t)pl.nx * pl.ny;
  g.gs = pl.nx;
  g.TA = pl.nx / g.W;
  g.TB = pl.ny / g.G;
  g.sa = g.W;
  g.sb = (int64_t)g.G * pl.nx;
  const int threads = 3 * g.W * g.G * TPL;
  const size_t smem = zcurl_tma_smem(L, g.W, g.G, S, sizeof(C));
  CUtensorMap m[3];
  for (int d = 0; d < 3; d++) {
    const int rc = field_tensor_map(&m[d], f.in[d], pl.nx, pl.ny, pl.nz, (int)sizeof(C), g.W,
                                    g.G, ZB);
    if (rc) return rc;
  }
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_zcurl_tma<T, L, S>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_zcurl_tma)");
    attr[dev & 63] = true;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zcurl_tma<T, L, S>,
                                                                threads, smem);
  if (e != cudaSuccess) return cuda_status(e, "occupancy(k_zcurl_tma)");
  if (per_sm < 1) {
    set_error("K1 TMA tile: does not fit on an SM");
    return ERR_UNSUPPORTED;
  }
  const int64_t ntiles = g.TA * g.TB;
  const int blocks = (int)std::min<int64_t>(ntiles, (int64_t)per_sm * sm_count());
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  int wshift = 0;
  while ((1 << wshift) < g.W) wshift++;
  e = launch_pdl(k_zcurl_tma<T, L, S>, dim3((unsigned)blocks), dim3(threads), smem, s, m[0], m[1],
                 m[2], g, f, tw, wshift, err, tma_stall_cycles());
  if (e != cudaSuccess) return cuda_status(e, "k_zcurl_tma");
  return OK;
}

template <typename T, int L>
int launch_zcurl(const NSPlan& pl, const FieldPtrs& f, int* err, cudaStream_t s) {
  if (pl.k1_tma && err)
    return pl.k1_stages == 1 ? launch_zcurl_tma<T, L, 1>(pl, f, err, s)
                             : launch_zcurl_tma<T, L, 2>(pl, f, err, s);
  return pl.k1_reload ? launch_zcurl_as<T, L, true>(pl, f, s)
                      : launch_zcurl_as<T, L, false>(pl, f, s);
}

template <typename T, int M>
int launch_xcross_r2c(const NSPlan& pl, const FieldPtrs& f, int64_t rows, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<M>::TPL;
  const int G = pl.xG;
  const int threads = 6 * G * TPL;
  const size_t smem = (size_t)6 * G * xrow_stride(M, (int)sizeof(C)) * sizeof(C);
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_xcross_r2c<T, M>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_xcross_r2c)");
    attr[dev & 63] = true;
  }
  const int prec = sizeof(T) == 8 ? PREC_C128 : PREC_C64;
  const C* twN = reinterpret_cast<const C*>(twiddles(2 * M, prec));
  const C* twM = reinterpret_cast<const C*>(twiddles(M, prec));
  if (!twN || !twM) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  const double N = (double)pl.nx_phys * pl.ny * pl.nz;
  cudaError_t e = launch_pdl(k_xcross_r2c<T, M>, dim3((unsigned)(rows / G)), dim3(threads), smem,
                             s, f, twN, twM, G, (T)(1.0 / (N * N)));
  if (e != cudaSuccess) return cuda_status(e, "k_xcross_r2c");
  return OK;
}

template <typename T>
int xcross_r2c(const NSPlan& pl, const FieldPtrs& f, int64_t rows, cudaStream_t s) {
  switch (pl.nx) {
    case 16: return launch_xcross_r2c<T, 16>(pl, f, rows, s);
    case 32: return launch_xcross_r2c<T, 32>(pl, f, rows, s);
    case 64: return launch_xcross_r2c<T, 64>(pl, f, rows, s);
    case 128: return launch_xcross_r2c<T, 128>(pl, f, rows, s);
    case 256: return launch_xcross_r2c<T, 256>(pl, f, rows, s);
    case 512: return launch_xcross_r2c<T, 512>(pl, f, rows, s);
    default: set_error("real-field NS step: nx must be a power of two in [32, 1024]"); return ERR_UNSUPPORTED;
  }
}

template <typename T>
int zcurl(const NSPlan& pl, const FieldPtrs& f, int* err, cudaStream_t s) {
  switch (pl.nz) {
    case 4: return launch_zcurl<T, 4>(pl, f, err, s);
    case 8: return launch_zcurl<T, 8>(pl, f, err, s);
    case 16: return launch_zcurl<T, 16>(pl, f, err, s);
    case 32: return launch_zcurl<T, 32>(pl, f, err, s);
    case 64: return launch_zcurl<T, 64>(pl, f, err, s);
    case 128: return launch_zcurl<T, 128>(pl, f, err, s);
    case 256: return launch_zcurl<T, 256>(pl, f, err, s);
    case 512: return launch_zcurl<T, 512>(pl, f, err, s);
    case 1024: return launch_zcurl<T, 1024>(pl, f, err, s);
    default: set_error("fused NS step: nz must be a power of two in [4, 1024]"); return ERR_UNSUPPORTED;
  }
}

template <typename T, int L, bool SGS>
int launch_update(const NSPlan& pl, const UpdateArgs& a, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  constexpr int NF = SGS ? 9 : 3;
  // a tile wider than the thread limit is z-transformed in two halves
  int threads = NF * a.W * TPL;
  if (threads > MaxThreads<T>::value && a.W % 2 == 0) threads /= 2;
  if (threads > MaxThreads<T>::value) {
    set_error("update pass: the tile width does not fit the thread limit");
    return ERR_ARG;
  }
  const size_t smem = (size_t)NF * a.W * tile_stride(L, a.W, (int)sizeof(C)) * sizeof(C);
  const int blocks = (int)(((int64_t)pl.nx * pl.ny) / a.W);
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_zfwd_update<T, L, SGS>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_zfwd_update)");
    attr[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  UpdateArgs ap = a;
  ap.pf = SGS ? 0 : tiles_in_waves(k_zfwd_update<T, L, SGS>, threads, smem, pl.pf_waves);
  ap.pf_self = SGS ? 0 : pl.z_pfself;
  cudaError_t e = launch_pdl(k_zfwd_update<T, L, SGS>, dim3(blocks), dim3(threads), smem, s, ap,
                             tw);
  if (e != cudaSuccess) return cuda_status(e, "k_zfwd_update");
  return OK;
}

// Shared memory of K5 with K1 carried: 3 W update rows, and 3 W exchange
// rows unless the new velocity is read back from V (reload).
inline size_t update_carry_smem(int L, int W, size_t esz, bool reload) {
  return (size_t)(reload ? 3 : 6) * W * tile_stride(L, W, (int)esz) * esz;
}

// Whether K5 with K1 carried can run W-line tiles on the box.
bool carry_ok(const NSPlan& p, int W, bool reload) {
  if (W > p.nx || p.nx % W) return false;
  const int TPL = p.nz >= 16 ? p.nz / 16 : 1;
  const size_t esz = p.prec == PREC_C128 ? 16 : 8;
  return 3 * W * TPL <= max_threads(p.prec) &&
         update_carry_smem(p.nz, W, esz, reload) <= 220 * 1024;
}

template <typename T, int L, bool RELOAD>
int launch_update_carry(const NSPlan& pl, const UpdateArgs& a, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  const int threads = 3 * a.W * TPL;
  const size_t smem = update_carry_smem(L, a.W, sizeof(C), RELOAD);
  const int blocks = (int)(((int64_t)pl.nx * pl.ny) / a.W);
  if (a.W > pl.nx || pl.nx % a.W || threads > MaxThreads<T>::value) {
    set_error("K5 with K1 carried: the tile width does not fit the box");
    return ERR_ARG;
  }
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_zfwd_update_curl<T, L, RELOAD>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_zfwd_update_curl)");
    attr[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  UpdateArgs ap = a;
  ap.pf = tiles_in_waves(k_zfwd_update_curl<T, L, RELOAD>, threads, smem, pl.pf_waves);
  ap.pf_self = pl.z_pfself;
  cudaError_t e =
      launch_pdl(k_zfwd_update_curl<T, L, RELOAD>, dim3(blocks), dim3(threads), smem, s, ap, tw);
  if (e != cudaSuccess) return cuda_status(e, "k_zfwd_update_curl");
  return OK;
}

// Shared memory of the TMA-staged K5: the stage (3 W x L boxes), 128 bytes of
// alignment slack, the 3 W padded rows and two mbarriers.
inline size_t update_tma_smem(int L, int W, size_t esz) {
  return ((size_t)3 * W * L + (size_t)3 * W * tile_stride(L, W, (int)esz)) * esz + 128 + 16;
}

// Whether the TMA-staged K5 can run W-line tiles on the box.
bool z_tma_ok(const NSPlan& p, int W) {
  if (p.nz < 16 || p.nz > 1024 || W > p.nx || p.nx % W) return false;
  const int TPL = p.nz / 16;
  const int esz = p.prec == PREC_C128 ? 16 : 8;
  return 3 * W * TPL <= max_threads(p.prec) && update_tma_smem(p.nz, W, esz) <= 220 * 1024 &&
         field_box_ok(p.nx, p.ny, p.nz, esz, W, 1, p.nz < 256 ? p.nz : 256);
}

template <typename T, int L>
int launch_update_tma(const NSPlan& pl, const UpdateArgs& a, int* err, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  constexpr int ZB = L < 256 ? L : 256;
  const int threads = 3 * a.W * TPL;
  const size_t smem = update_tma_smem(L, a.W, sizeof(C));
  CUtensorMap m[3];
  for (int d = 0; d < 3; d++) {
    const int rc = field_tensor_map(&m[d], a.U[d], pl.nx, pl.ny, pl.nz, (int)sizeof(C), a.W, 1, ZB);
    if (rc) return rc;
  }
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_zfwd_update_tma<T, L>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_zfwd_update_tma)");
    attr[dev & 63] = true;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zfwd_update_tma<T, L>,
                                                                threads, smem);
  if (e != cudaSuccess) return cuda_status(e, "occupancy(k_zfwd_update_tma)");
  if (per_sm < 1) {
    set_error("K5 TMA tile: does not fit on an SM");
    return ERR_UNSUPPORTED;
  }
  const int64_t ntiles = ((int64_t)pl.nx * pl.ny) / a.W;
  const int blocks = (int)std::min<int64_t>(ntiles, (int64_t)per_sm * sm_count());
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  e = launch_pdl(k_zfwd_update_tma<T, L>, dim3((unsigned)blocks), dim3(threads), smem, s, m[0],
                 m[1], m[2], a, tw, ntiles, err, tma_stall_cycles());
  if (e != cudaSuccess) return cuda_status(e, "k_zfwd_update_tma");
  return OK;
}

template <typename T>
int xcross(const NSPlan& pl, const FieldPtrs& f, int64_t rows, int* err, cudaStream_t s) {
  const bool tma = pl.x_tma && err;
  switch (pl.nx) {
#define SNS_XCROSS_CASE(L)                                                                   \
  case L:                                                                                    \
    return tma ? launch_xcross_tma<T, L>(pl, f, rows, err, s) : launch_xcross<T, L>(pl, f, rows, s);
    SNS_XCROSS_CASE(4)
    SNS_XCROSS_CASE(8)
    SNS_XCROSS_CASE(16)
    SNS_XCROSS_CASE(32)
    SNS_XCROSS_CASE(64)
    SNS_XCROSS_CASE(128)
    SNS_XCROSS_CASE(256)
    SNS_XCROSS_CASE(512)
    SNS_XCROSS_CASE(1024)
#undef SNS_XCROSS_CASE
    default: set_error("fused NS step: nx must be a power of two in [4, 1024]"); return ERR_UNSUPPORTED;
  }
}

template <typename T, bool SGS>
int update(const NSPlan& pl, const UpdateArgs& a, int* err, cudaStream_t s) {
  const bool tma = !SGS && pl.z_tma && err;
  switch (pl.nz) {
#define SNS_UPDATE_CASE(L)                                                                   \
  case L:                                                                                    \
    if constexpr (L >= 16) {                                                                 \
      if (tma) return launch_update_tma<T, L>(pl, a, err, s);                                \
    }                                                                                        \
    return launch_update<T, L, SGS>(pl, a, s);
    SNS_UPDATE_CASE(4)
    SNS_UPDATE_CASE(8)
    SNS_UPDATE_CASE(16)
    SNS_UPDATE_CASE(32)
    SNS_UPDATE_CASE(64)
    SNS_UPDATE_CASE(128)
    SNS_UPDATE_CASE(256)
    SNS_UPDATE_CASE(512)
    SNS_UPDATE_CASE(1024)
#undef SNS_UPDATE_CASE
    default: set_error("fused NS step: nz must be a power of two in [4, 1024]"); return ERR_UNSUPPORTED;
  }
}

template <typename T>
int update_carry(const NSPlan& pl, const UpdateArgs& a, cudaStream_t s) {
  const bool r = pl.carry_reload;
  switch (pl.nz) {
#define SNS_CARRY_CASE(L)                                                                    \
  case L:                                                                                    \
    return r ? launch_update_carry<T, L, true>(pl, a, s) : launch_update_carry<T, L, false>(pl, a, s);
    SNS_CARRY_CASE(4)
    SNS_CARRY_CASE(8)
    SNS_CARRY_CASE(16)
    SNS_CARRY_CASE(32)
    SNS_CARRY_CASE(64)
    SNS_CARRY_CASE(128)
    SNS_CARRY_CASE(256)
    SNS_CARRY_CASE(512)
    SNS_CARRY_CASE(1024)
#undef SNS_CARRY_CASE
    default: set_error("fused NS step: nz must be a power of two in [4, 1024]"); return ERR_UNSUPPORTED;
  }
}

// K3 of the plan: complex rows, or half-spectrum rows of a real-field run
int xpass(const NSPlan& pl, const FieldPtrs& f, int64_t rows, int* err, cudaStream_t s) {
  if (pl.real)
    return pl.prec == PREC_C128 ? xcross_r2c<double>(pl, f, rows, s)
                                : xcross_r2c<float>(pl, f, rows, s);
  return pl.prec == PREC_C128 ? xcross<double>(pl, f, rows, err, s)
                              : xcross<float>(pl, f, rows, err, s);
}

int elems(int L) { return L >= 16 ? 16 : L; }

}  // namespace

int ns_plan(NSPlan& pl, int nx, int ny, int nz, int prec, int zW, int lineW, bool real) {
  pl = NSPlan{};
  pl.real = real;
  pl.nx_phys = nx;
  if (real) {
    // half spectrum: kx = 0 .. nx/2-1 stored (the kx = nx/2 plane is zero)
    if (!is_pow2(nx) || nx < 32 || nx > 1024) {
      set_error("real-field NS step: nx must be a power of two in [32, 1024]");
      return ERR_UNSUPPORTED;
    }
    nx /= 2;
  }
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
           (size_t)6 * G * 2 * xrow_stride(nx, (int)esz) * esz <= 110 * 1024)
      G *= 2;
    if (6 * G * TPL > max_threads(prec)) {
      set_error("fused NS step: nx too large for the x-pass tile");
      return ERR_UNSUPPORTED;
    }
    pl.xG = G;
    // the TMA-staged form on request (SNS_X_TMA=1), with the widest tile up
    // to G that fits its stage.  Measured on B200 at 256^3 it does not pay:
    // complex64 0.315 ms against 0.284 (G = 4) and 0.262 (G = 2, direct);
    // complex128 0.700 against 0.756 (G = 4) and 0.599 (G = 1, direct): the
    // rows are contiguous, so direct loads already stream, and the stage
    // halves the CTAs an SM holds.  The tuner still tries it.
    // the five-CTA form of the direct-load pass on request (SNS_X_OCC=1)
    const char* eo = getenv("SNS_X_OCC");
    pl.x_occ = eo && eo[0] == '1';
    const char* e = getenv("SNS_X_TMA");
    pl.x_tma = false;
    if (e && e[0] == '1')
      for (int g = G; g >= 1 && !pl.x_tma; g /= 2)
        if (x_tma_ok(pl, g)) {
          pl.x_tma = true;
          pl.xG = g;
        }
  }
  // K1 tile: W adjacent z lines x G groups of the three components, one
  // CTA for all six outputs (SNS_K1_SPLIT=1: one output field per CTA)
  {
    // 16 adjacent lines keep the half-warps of the exchanges on distinct banks;
    // the two row sets of a 16-line tile take 210 KB at 256 (opt-in limit 227 KB)
    // Two CTAs per SM (112 KB each), so that one CTA's loads overlap the
    // other's transforms; tile_stride keeps narrower runs free of bank
    // conflicts.  SNS_K1_SMEM_KB overrides the cap (220: one CTA per SM).
    const int TPL = nz / elems(nz);
    const int cap = max_threads(prec);
    size_t smem_cap = 112 * 1024;
    if (const char* e = getenv("SNS_K1_SMEM_KB")) {
      const int v = atoi(e);
      if (v >= 16 && v <= 220) smem_cap = (size_t)v * 1024;
    }
    int W = 1;
    const int Wmax = prec == PREC_C128 ? 8 : 16;
    while (W * 2 <= Wmax && nx % (W * 2) == 0 && 3 * (W * 2) * TPL <= cap &&
           (size_t)6 * (W * 2) * tile_stride(nz, W * 2, (int)esz) * esz <= smem_cap)
      W *= 2;
    int G = 1;
    while (ny % (G * 2) == 0 && 3 * W * (G * 2) * TPL <= 384 &&
           (size_t)6 * W * (G * 2) * tile_stride(nz, W, (int)esz) * esz <= smem_cap)
      G *= 2;
    pl.k1W = W;
    pl.k1G = G;
    const char* e = getenv("SNS_K1_SPLIT");
    pl.k1_fused = !(e && e[0] == '1') && 3 * W * G * TPL <= cap &&
                  (size_t)6 * W * G * tile_stride(nz, W, (int)esz) * esz <= smem_cap;
  }
  // K5 tile: W adjacent z lines of three fields
  {
    const int TPL = nz / elems(nz);
    int W = 1;
    int Wmax = prec == PREC_C128 ? 8 : 16;
    if (zW > 0) Wmax = zW;  // a tuned width
    // tile width override for tuning sweeps (SNS_Z_W, a power of two; a
    // width beyond the thread limit is transformed in two halves, with one
    // CTA per SM)
    bool wide = false;
    if (const char* e = zW > 0 ? nullptr : getenv("SNS_Z_W")) {
      const int v = atoi(e);
      if (v >= 1 && (v & (v - 1)) == 0) Wmax = v;
      wide = true;
    }
    while (W * 2 <= Wmax && nx % (W * 2) == 0 &&
           3 * (W * 2) * TPL <= (wide ? 2 : 1) * max_threads(prec) &&
           (size_t)3 * W * 2 * tile_stride(nz, W * 2, (int)esz) * esz <= (wide ? 220 : 110) * 1024)
      W *= 2;
    pl.zW = W;
    pl.update_blocks = (nx / W) * ny;
    // the TMA-staged form on request (SNS_Z_TMA=1), the widest tile up to W
    // that fits its stage.  Measured on B200 at 256^3 it does not pay: complex64
    // 0.500 ms (W = 16) and 0.657 (W = 8) against 0.435 direct; complex128
    // 1.159 (W = 8) against 1.016.  The cross product is only a third of the
    // pass's reads (V and C0 load in the update), the stage and the rows fill
    // the SM's shared memory at one CTA, and the persistent tiles add two
    // barriers each.  The tuner still tries it.
    const char* ez = getenv("SNS_Z_TMA");
    pl.z_tma = false;
    if (ez && ez[0] == '1')
      for (int w = W; w >= 1 && !pl.z_tma; w /= 2)
        if (z_tma_ok(pl, w)) {
          pl.z_tma = true;
          pl.zW = w;
          pl.update_blocks = (nx / w) * ny;
        }
    // K1 carried in the update pass on request (SNS_CARRY=1), at the widest
    // tile up to W whose update and exchange rows fit two CTAs per SM
    // (SNS_CARRY=2: the new velocity read back from V, K5's shared memory)
    const char* ecr = getenv("SNS_CARRY");
    pl.carry = false;
    pl.carry_reload = ecr && ecr[0] == '2';
    if (ecr && (ecr[0] == '1' || ecr[0] == '2'))
      for (int w = W; w >= 1 && !pl.carry; w /= 2)
        if (carry_ok(pl, w, pl.carry_reload) &&
            update_carry_smem(nz, w, esz, pl.carry_reload) <= 110 * 1024) {
          pl.carry = true;
          pl.z_tma = false;
          pl.zW = w;
          pl.update_blocks = (nx / w) * ny;
        }
    // L2 prefetch of each tile's V and C0 once its cross product's loads are
    // in flight (SNS_Z_PFSELF=1; asked before those loads it delayed them and
    // measured slower)
    const char* epf = getenv("SNS_Z_PFSELF");
    pl.z_pfself = epf && epf[0] == '1';
    // closure update: nine fields in the tile
    const int cap = std::min(576, max_threads(prec));
    int Ws = 1;
    while (Ws * 2 <= Wmax && ((int64_t)nx * ny) % (Ws * 2) == 0 && 9 * (Ws * 2) * TPL <= cap &&
           (size_t)9 * Ws * 2 * tile_stride(nz, Ws * 2, (int)esz) * esz <= 110 * 1024)
      Ws *= 2;
    pl.sgs_W = Ws;
    pl.sgs_blocks = (int)(((int64_t)nx * ny) / Ws);
  }
  // xy phase: three separate full-domain passes by default.  Two fused forms
  // move a third of their HBM bytes but measured slower on B200, the passes
  // being bound by latency and issue rather than bytes: SNS_XYC=1 selects one
  // thread-block-cluster pass over each plane (sns_xyc.cu; nx = ny = 128, or
  // 256 in complex64; 1.28 vs 0.73 ms at 256^3), SNS_XY_PASSES=1 the
  // persistent dataflow launch through L2 (sns_xy.cu; 1.09 vs 0.79 ms).
  const char* env = getenv("SNS_XY_PASSES");
  const bool dataflow = env && env[0] == '1';
  pl.use_xy = !real && dataflow && xy_supported(nx, ny, prec) &&
              xy_plan(pl.xy, nx, ny, nz, prec) == OK;
  pl.use_xyc = !real && !pl.use_xy && xyc_supported(nx, ny, prec);
  // separate passes run in slabs of xy_chunk planes (SNS_XY_CHUNK; 0 = one slab)
  pl.xy_chunk = 0;
  if (const char* e = getenv("SNS_XY_CHUNK")) pl.xy_chunk = atoi(e);
  if (pl.xy_chunk > 0 && pl.xy_chunk < nz) pl.use_xyc = false;
  pl.passes = (pl.use_xy || pl.use_xyc || (pl.xy_chunk > 0 && pl.xy_chunk < nz)) ? 3 : 5;
  pl.lineW = lineW > 0 ? lineW : 0;
  pl.lineT = 0;
  pl.lineOrd = 0;
  {
    // the y passes over TMA-staged tiles on request (SNS_Y_TMA = 1 or 2 stages)
    const char* e = getenv("SNS_Y_TMA");
    const int v = e ? atoi(e) : 0;
    pl.y_tma = 0;
    if ((v == 1 || v == 2) && line_tma_ok(axis_geo(1, nx, ny, nz, prec), prec, v))
      pl.y_tma = v;
  }
  pl.tuned = false;
  pl.k1_lines = false;  // enabled by a caller that provides the work fields W
  {
    // L2 prefetch of the tile a wave or two ahead (SNS_PF = 0, 1, 2 waves)
    const char* e = getenv("SNS_PF");
    pl.pf_waves = e ? std::max(0, std::min(4, atoi(e))) : 0;
  }
  {
    const char* e = getenv("SNS_K1_RELOAD");
    pl.k1_reload = e && e[0] == '1';
  }
  {
    // K1 over TMA-staged tiles, one stage by default (SNS_K1_TMA = 0: off,
    // 2: two stages); an explicit SNS_K1_RELOAD=1 or SNS_K1_SPLIT=1 keeps
    // that form.  Measured on B200 at 256^3: complex64 0.28 ms against 0.37
    // (reload tile), complex128 0.58 against 0.79 (split).
    const char* e = getenv("SNS_K1_TMA");
    const char* es = getenv("SNS_K1_SPLIT");
    const int v = e ? atoi(e) : ((pl.k1_reload || (es && es[0] == '1')) ? 0 : 1);
    pl.k1_stages = v == 2 ? 2 : 1;
    pl.k1_tma = false;
    if (v == 1 || v == 2) {
      // the widest tile of at most 384 threads that fits the stages
      const int TPL = nz / elems(nz);
      for (int W = 16; W >= 1 && !pl.k1_tma; W /= 2)
        for (int G = 4; G >= 1 && !pl.k1_tma; G /= 2)
          if (3 * W * G * TPL <= 384 && k1_tma_ok(pl, W, G, pl.k1_stages)) {
            pl.k1_tma = true;
            pl.k1_fused = true;
            pl.k1W = W;
            pl.k1G = G;
          }
    }
  }
  pl.k1lW = 0;
  pl.k1lT = 0;
  pl.kc2 = 1e300;
  pl.sgs_klo = 0;
  pl.sgs_kinv = 1e30;
  return OK;
}

namespace {

// K1 as a z pass of V into U[0..5] (the fused tile or one field per CTA).
int run_k1(const NSPlan& pl, void* const V[3], void* const U[6], int* err_word, cudaStream_t s) {
  FieldPtrs f{};
  f.n = 6;
  for (int d = 0; d < 3; d++) f.in[d] = V[d];
  for (int i = 0; i < 6; i++) f.out[i] = U[i];
  if (pl.k1_fused)
    return pl.prec == PREC_C128 ? zcurl<double>(pl, f, err_word, s)
                                : zcurl<float>(pl, f, err_word, s);
  LineGeo g = axis_geo(2, pl.nx, pl.ny, pl.nz, pl.prec, pl.lineW);
  g.kx_half = pl.real;
  return run_line_pass(g, f, +1, 0, 1.0, pl.prec, s, PRO_CURL6);
}

}  // namespace

int ns_k1_once(const NSPlan& pl, void* const V[3], void* const U[6], int* sync_words,
               cudaStream_t s) {
  if (pl.k1_lines) {
    set_error("ns_k1_once: K1 as a line pass writes the work fields W, not U");
    return ERR_ARG;
  }
  return run_k1(pl, V, U, sync_words ? sync_words + xy_sync_words(pl.nz) - 1 : nullptr, s);
}

int ns_step_once(const NSPlan& pl, void* const V[3], void* const C0[3], void* const U[6],
                 double* stats, int* sync_words, double nu, double dt, cudaStream_t s,
                 cudaEvent_t* ev, void* const* W, bool* carried) {
  const int nx = pl.nx, ny = pl.ny, nz = pl.nz, prec = pl.prec;
  // the error word of the step's bounded waits
  int* err_word = sync_words ? sync_words + xy_sync_words(nz) - 1 : nullptr;
  int rc;
  int pass = 0;
  auto mark = [&]() {
    if (ev) cudaEventRecord(ev[pass], s);
    pass++;
  };
  mark();
  const bool lines = pl.k1_lines && W && !pl.use_xy && !pl.use_xyc;
  // K1 carried in the previous step's K5: U already holds its output
  const bool carry = pl.carry && carried && !lines;
  const bool have_k1 = carry && *carried;
  if (carried) *carried = false;
  // K1: z-inverse of (V, i k x V)
  if (have_k1) {
    mark();
  } else if (lines) {
    // V and the z derivatives i kz Vx, i kz Vy (taken on the way in), each
    // field z-inverse-transformed on its own; K2 forms omega from them
    FieldPtrs f{};
    f.n = kNSLineWork;
    for (int d = 0; d < 3; d++) f.in[d] = V[d];
    f.in[3] = V[0];
    f.in[4] = V[1];
    for (int i = 0; i < kNSLineWork; i++) f.out[i] = W[i];
    f.ikmask = 0x18u;
    LineGeo g = axis_geo(2, nx, ny, nz, prec, pl.k1lW, pl.k1lT);
    g.kx_half = pl.real;
    rc = run_line_pass(g, f, +1, 0, 1.0, prec, s, PRO_IKAXIS);
    if (rc) return rc;
    mark();
  } else {
    if ((rc = run_k1(pl, V, U, err_word, s))) return rc;
    mark();
  }
  if (pl.use_xy) {
    // K2 + K3 + K4 as one persistent dataflow launch (sns_xy.cu)
    if ((rc = xy_run(pl.xy, U, sync_words, s))) return rc;
    mark();
  } else if (pl.use_xyc) {
    // K2 + K3 + K4 as one cluster pass over each plane (sns_xyc.cu)
    if ((rc = xyc_run(U, nx, ny, nz, prec, s))) return rc;
    mark();
  }
  // K2, K3, K4 on the planes [z0, z0 + pz): the passes treat the slab as an
  // nx*ny*pz field at an offset pointer (the 1/N^2 scale keeps the full N)
  const size_t esz = prec == PREC_C128 ? 16 : 8;
  auto xy_range = [&](int z0, int pz, bool marks) -> int {
    const size_t off = esz * (size_t)z0 * nx * ny;
    void* Uc[6];
    for (int i = 0; i < 6; i++) Uc[i] = static_cast<char*>(U[i]) + off;
    if (lines) {  // K2: y-inverse of V and of omega formed from the five z-inverted fields
      FieldPtrs f{};
      f.n = 6;
      for (int i = 0; i < kNSLineWork; i++) f.in[i] = static_cast<char*>(W[i]) + off;
      f.in[5] = f.in[0];
      for (int i = 0; i < 6; i++) f.out[i] = Uc[i];
      LineGeo g = axis_geo(1, nx, ny, pz, prec, pl.lineW, pl.lineT, pl.lineOrd);
      g.kx_half = pl.real;
      g.pfw = pl.pf_waves;
      int r = run_line_pass(g, f, +1, 0, 1.0, prec, s, PRO_OMEGA);
      if (r) return r;
      if (marks) mark();
    } else {  // K2: y-inverse of the six fields
      FieldPtrs f{};
      f.n = 6;
      for (int i = 0; i < 6; i++) f.in[i] = f.out[i] = Uc[i];
      LineGeo g = axis_geo(1, nx, ny, pz, prec, pl.lineW, pl.lineT, pl.lineOrd);
      g.pfw = pl.pf_waves;
      int r = pl.y_tma && err_word && line_tma_ok(g, prec, pl.y_tma)
                  ? run_line_pass_tma(g, f, +1, 0, 1.0, prec, s, pl.y_tma, err_word)
                  : run_line_pass(g, f, +1, 0, 1.0, prec, s);
      if (r) return r;
      if (marks) mark();
    }
    {  // K3: x-inverse, cross product, x-forward
      FieldPtrs f{};
      f.n = 6;
      for (int i = 0; i < 6; i++) f.in[i] = Uc[i];
      for (int i = 0; i < 3; i++) f.out[i] = Uc[i];
      const int64_t rows = (int64_t)ny * pz;
      int r = xpass(pl, f, rows, err_word, s);
      if (r) return r;
      if (marks) mark();
    }
    {  // K4: y-forward of the cross product
      FieldPtrs f{};
      f.n = 3;
      for (int i = 0; i < 3; i++) f.in[i] = f.out[i] = Uc[i];
      LineGeo g = axis_geo(1, nx, ny, pz, prec, pl.lineW, pl.lineT, pl.lineOrd);
      g.pfw = pl.pf_waves;
      int r = pl.y_tma && err_word && line_tma_ok(g, prec, pl.y_tma)
                  ? run_line_pass_tma(g, f, -1, 0, 1.0, prec, s, pl.y_tma, err_word)
                  : run_line_pass(g, f, -1, 0, 1.0, prec, s);
      if (r) return r;
    }
    return OK;
  };
  if (!pl.use_xy && !pl.use_xyc) {
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
    a.lx = 0;
    while ((1 << a.lx) < nx) a.lx++;
    a.hK = dt / 2;
    a.nuhK = nu * dt / 2;
    a.stats = stats;
    a.kc2 = pl.kc2;
    a.kx_half = pl.real;
    if (carry) {
      // K5 with the next step's K1 carried: U receives the z-inverse of the
      // new V and of its curl
      for (int i = 0; i < 6; i++) a.Uo[i] = U[i];
      rc = prec == PREC_C128 ? update_carry<double>(pl, a, s) : update_carry<float>(pl, a, s);
    } else {
      rc = ns_update(pl, a, false, s, err_word);
    }
    if (rc) return rc;
    if (carried) *carried = carry;
    mark();
  }
  return OK;
}

namespace {

constexpr size_t kTuneSmemCap = 220 * 1024;

// Seeded values in [-1, 1) for the tuner's timing steps, so that every pass
// runs on data of the magnitude a run has (a counter hash, not a statistical
// generator).
template <typename T>
__global__ void k_fill_tune(cx_t<T>* p, int64_t n, uint32_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t h = (uint32_t)i * 2654435761u ^ seed;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    const uint32_t h2 = h * 3266489917u ^ (h >> 16);
    p[i] = mk((T)((int32_t)h) * (T)4.656612873077393e-10,
              (T)((int32_t)h2) * (T)4.656612873077393e-10);
  }
}

int fill_tune(void* p, int64_t n, int prec, uint32_t seed, cudaStream_t s) {
  const int grid = std::max(1, std::min(4 * sm_count(), (int)((n + 255) / 256)));
  if (prec == PREC_C128)
    k_fill_tune<double><<<grid, 256, 0, s>>>(reinterpret_cast<double2*>(p), n, seed);
  else
    k_fill_tune<float><<<grid, 256, 0, s>>>(reinterpret_cast<float2*>(p), n, seed);
  SNS_CHECK_LAUNCH("k_fill_tune");
  return OK;
}

bool k1_ok(const NSPlan& p, int W, int G, bool reload) {
  const int TPL = p.nz / elems(p.nz);
  const size_t esz = p.prec == PREC_C128 ? 16 : 8;
  return p.nx % W == 0 && p.ny % G == 0 && 3 * W * G * TPL <= max_threads(p.prec) &&
         (size_t)(reload ? 3 : 6) * W * G * tile_stride(p.nz, W, (int)esz) * esz <= kTuneSmemCap;
}
bool xg_ok(const NSPlan& p, int G) {
  const int TPL = p.nx / elems(p.nx);
  const size_t esz = p.prec == PREC_C128 ? 16 : 8;
  const int cap = p.real ? 384 : max_threads(p.prec);  // k_xcross_r2c launch bound
  return ((int64_t)p.ny * p.nz) % G == 0 && 6 * G * TPL <= cap &&
         (size_t)6 * G * xrow_stride(p.nx, (int)esz) * esz <= kTuneSmemCap;
}
bool zw_ok(const NSPlan& p, int W, int max_blocks, bool halves = false) {
  const int TPL = p.nz / elems(p.nz);
  const size_t esz = p.prec == PREC_C128 ? 16 : 8;
  // halves: the plain update pass may transform a tile in two halves of W/2
  const int thr = 3 * W * TPL / (halves && 3 * W * TPL > max_threads(p.prec) ? 2 : 1);
  return p.nx % W == 0 && thr <= max_threads(p.prec) &&
         (size_t)3 * W * tile_stride(p.nz, W, (int)esz) * esz <= kTuneSmemCap &&
         ((int64_t)p.nx * p.ny) / W <= max_blocks;
}

}  // namespace

int ns_tune_plan(NSPlan& pl, void* const V[3], void* const C0[3], void* const U[6],
                 double* stats, int max_blocks, int* sync_words, cudaStream_t s,
                 void* const* W) {
  if (pl.passes != kNSPasses) return OK;
  cudaEvent_t ev[kNSPasses + 1];
  int rc = OK;
  // the timing steps run on seeded data (with dt = 0 and nu = 0 a step only
  // projects V, so the values stay bounded); the caller clears them after
  const int64_t n = (int64_t)pl.nx * pl.ny * pl.nz;
  for (int d = 0; d < 3 && rc == OK; d++) {
    rc = fill_tune(V[d], n, pl.prec, 17u + d, s);
    if (rc == OK) rc = fill_tune(C0[d], n, pl.prec, 29u + d, s);
  }
  int made = 0;
  for (; made < kNSPasses + 1 && rc == OK; made++)
    rc = cuda_status(cudaEventCreate(&ev[made]), "ns_tune_plan(events)");
  // time of the passes in the bit mask `passes` of a candidate plan: one step
  // to set the kernels up, then the least of five timed steps
  auto measure = [&](const NSPlan& c, unsigned passes, float* out) -> int {
    float best = 3.4e38f;
    bool carried = false;
    for (int r = 0; r < 6; r++) {
      int e = ns_step_once(c, V, C0, U, stats, sync_words, 0.0, 0.0, s, r ? ev : nullptr, W,
                           &carried);
      if (e) return e;
      if (!r) continue;
      if ((e = cuda_status(cudaEventSynchronize(ev[kNSPasses]), "ns_tune_plan"))) return e;
      float sum = 0;
      for (int p = 0; p < kNSPasses; p++)
        if ((passes >> p) & 1u) {
          float t = 0;
          cudaEventElapsedTime(&t, ev[p], ev[p + 1]);
          sum += t;
        }
      best = std::min(best, sum);
    }
    *out = best;
    return OK;
  };
  // SNS_TUNE_LOG=1 prints every candidate's time to stderr
  const bool log = getenv("SNS_TUNE_LOG") && getenv("SNS_TUNE_LOG")[0] == '1';
  // margin > 0: cands[0] is the incumbent plan, and another candidate
  // replaces it only when faster by that fraction (whole-step timings of a few
  // steps vary by 1-2 % between runs)
  auto pick = [&](std::vector<NSPlan>& cands, unsigned passes, float margin = 0.f) -> int {
    float best = 3.4e38f, t0 = 3.4e38f;
    int bi = -1;
    for (size_t i = 0; i < cands.size(); i++) {
      float t = 0;
      int e = measure(cands[i], passes, &t);
      if (e) return e;
      if (log)
        fprintf(stderr,
                "ns_tune passes=0x%x cand=%zu ms=%.4f k1=%dx%d%s%s xG=%d%s zW=%d%s%s lineW=%d "
                "lineT=%d ord=%d ytma=%d pf=%d\n",
                passes, i, t, cands[i].k1W, cands[i].k1G, cands[i].k1_tma ? "(tma)" : "",
                cands[i].k1_reload ? "(reload)" : "", cands[i].xG,
                cands[i].x_tma ? "(tma)" : cands[i].x_occ ? "(occ)" : "",
                cands[i].zW, cands[i].z_tma ? "(tma)" : cands[i].z_pfself ? "(pfs)" : "",
                cands[i].carry ? (cands[i].carry_reload ? "(+K1r)" : "(+K1)") : "",
                cands[i].lineW, cands[i].lineT, cands[i].lineOrd, cands[i].y_tma,
                cands[i].pf_waves);
      if (i == 0) t0 = t;
      if (t < best) {
        best = t;
        bi = (int)i;
      }
    }
    if (margin > 0.f && bi > 0 && best > t0 * (1.f - margin)) bi = 0;
    if (bi >= 0) pl = cands[bi];
    return OK;
  };
  std::vector<NSPlan> c;
  // K1: the z-inverse + curl pass as a fused tile (its shape), one output
  // field per CTA, or the five-field line pass with the curl formed in K2
  // (its run width and thread cap); timed with K2, whose input it sets
  if (rc == OK) {
    c.clear();
    c.push_back(pl);
    for (int reload = 0; reload < 2; reload++)
      for (int Wd : {2, 4, 8, 16})
        for (int G : {1, 2, 4})
          if (k1_ok(pl, Wd, G, reload)) {
            NSPlan q = pl;
            q.k1W = Wd;
            q.k1G = G;
            q.k1_fused = true;
            q.k1_reload = reload;
            q.k1_lines = false;
            q.k1_tma = false;
            c.push_back(q);
          }
    // the persistent pass over TMA-staged tiles (one or two stages)
    if (sync_words)
      for (int S = 1; S <= 2; S++)
        for (int Wd : {2, 4, 8, 16})
          for (int G : {1, 2, 4})
            if (k1_tma_ok(pl, Wd, G, S)) {
              NSPlan q = pl;
              q.k1W = Wd;
              q.k1G = G;
              q.k1_fused = true;
              q.k1_tma = true;
              q.k1_stages = S;
              q.k1_lines = false;
              c.push_back(q);
            }
    NSPlan split = pl;
    split.k1_fused = false;
    split.k1_lines = false;
    split.k1_tma = false;
    c.push_back(split);
    if (W)
      for (int Wd : {8, 16})
        for (int T : {256, 512}) {
          NSPlan q = pl;
          q.k1_lines = true;
          q.k1_tma = false;
          q.k1lW = Wd;
          q.k1lT = T;
          c.push_back(q);
        }
    rc = pick(c, 0x3u);
  }
  // K2 + K4: run width and thread cap, then radix order, of the y line passes
  if (rc == OK) {
    c.clear();
    for (int W : {4, 8, 16, 32})
      for (int T : {128, 256, 512})
        for (int S = 0; S <= (sync_words ? 2 : 0); S++) {
          NSPlan q = pl;
          q.lineW = W;
          q.lineT = T;
          q.y_tma = S;
          if (S && !line_tma_ok(axis_geo(1, pl.nx, pl.ny, pl.nz, pl.prec, W, T, pl.lineOrd),
                                pl.prec, S))
            continue;
          c.push_back(q);
        }
    rc = pick(c, 0xAu);
  }
  if (rc == OK && pl.ny >= 64 && pl.ny <= 1024) {
    c.clear();
    for (int o = 0; o < kRadixOrders; o++) {
      NSPlan q = pl;
      q.lineOrd = o;
      if (q.y_tma && !line_tma_ok(axis_geo(1, pl.nx, pl.ny, pl.nz, pl.prec, pl.lineW, pl.lineT, o),
                                  pl.prec, q.y_tma))
        continue;
      c.push_back(q);
    }
    rc = pick(c, 0xAu);
  }
  // K3: rows per CTA of the x cross pass
  if (rc == OK) {
    c.clear();
    for (int G : {1, 2, 4, 8, 16}) {
      if (xg_ok(pl, G)) {
        NSPlan q = pl;
        q.xG = G;
        q.x_tma = false;
        q.x_occ = false;
        c.push_back(q);
        // the five-CTA form, for CTAs of at most 192 threads (complex64)
        if (!pl.real && pl.prec == PREC_C64 && 6 * G * (pl.nx / elems(pl.nx)) <= 192) {
          q.x_occ = true;
          c.push_back(q);
        }
      }
      if (sync_words && x_tma_ok(pl, G)) {
        NSPlan q = pl;
        q.xG = G;
        q.x_occ = false;
        q.x_tma = true;
        c.push_back(q);
      }
    }
    if (!c.empty()) rc = pick(c, 0x4u);
  }
  // K5: adjacent z lines per CTA of the update pass
  if (rc == OK) {
    c.clear();
    for (int W : {2, 4, 8, 16, 32, 64}) {
      if (zw_ok(pl, W, max_blocks, true))
        for (int pfs = 0; pfs < 2; pfs++) {
          NSPlan q = pl;
          q.zW = W;
          q.z_tma = false;
          q.z_pfself = pfs == 1;
          q.update_blocks = (pl.nx / W) * pl.ny;
          c.push_back(q);
        }
      if (sync_words && zw_ok(pl, W, max_blocks) && z_tma_ok(pl, W)) {
        NSPlan q = pl;
        q.zW = W;
        q.z_tma = true;
        q.update_blocks = (pl.nx / W) * pl.ny;
        c.push_back(q);
      }
    }
    if (!c.empty()) rc = pick(c, 0x10u);
  }
  // K5 with the next step's K1 carried in it (tile widths), against the
  // plan so far, over the whole step: it trades K1's pass for a heavier K5.
  // Measured slower in steady state on B200 at 256^3 (whole step 1.53 against
  // 1.45 ms, and 0.78 against 0.71 ms for K5 + K1 in a long run), so it is
  // only tried on request (SNS_TUNE_CARRY=1)
  const char* etc = getenv("SNS_TUNE_CARRY");
  if (rc == OK && !pl.k1_lines && !getenv("SNS_CARRY") && etc && etc[0] == '1') {
    c.clear();
    c.push_back(pl);
    for (int reload = 0; reload < 2; reload++)
      for (int Wd : {2, 4, 8, 16, 32})
        if (zw_ok(pl, Wd, max_blocks) && carry_ok(pl, Wd, reload)) {
          NSPlan q = pl;
          q.carry = true;
          q.carry_reload = reload;
          q.z_tma = false;
          q.zW = Wd;
          q.update_blocks = (pl.nx / Wd) * pl.ny;
          c.push_back(q);
        }
    rc = pick(c, 0x1Fu, 0.02f);
  }
  // L2 prefetch distance of all five passes, timed over the whole step
  // (unless SNS_PF fixes it)
  if (rc == OK && !getenv("SNS_PF")) {
    c.clear();
    c.push_back(pl);
    for (int pw : {0, 1, 2}) {
      if (pw == pl.pf_waves) continue;
      NSPlan q = pl;
      q.pf_waves = pw;
      c.push_back(q);
    }
    rc = pick(c, 0x1Fu, 0.02f);
  }
  for (int i = 0; i < made; i++) cudaEventDestroy(ev[i]);
  if (rc == OK) pl.tuned = true;
  return rc;
}

int ns_update(const NSPlan& pl, const UpdateArgs& a, bool sgs, cudaStream_t s, int* err) {
  if (pl.prec == PREC_C128)
    return sgs ? update<double, true>(pl, a, err, s) : update<double, false>(pl, a, err, s);
  return sgs ? update<float, true>(pl, a, err, s) : update<float, false>(pl, a, err, s);
}

// The normalisation sns_ns_stats applies on the host (mean |div|, 1/2 <|u|^2>,
// 1/2 <|omega|^2> of the unnormalised Fourier fields), with the same divisions.
__global__ void k_stats_normalise(double* out4, double N) {
  if (threadIdx.x == 0) {
    out4[0] = out4[0] / N;
    out4[1] = 0.5 * out4[1] / (N * N);
    out4[2] = 0.5 * out4[2] / (N * N);
  }
}

int ns_stats_normalise(double* out4, double N, cudaStream_t s) {
  k_stats_normalise<<<1, 32, 0, s>>>(out4, N);
  SNS_CHECK_LAUNCH("k_stats_normalise");
  return OK;
}

int ns_stats_final(const double* partials, int blocks, double* out4, cudaStream_t s) {
  k_stats_final<<<1, 256, 0, s>>>(partials, blocks, out4);
  SNS_CHECK_LAUNCH("k_stats_final");
  return OK;
}

}  // namespace sns
