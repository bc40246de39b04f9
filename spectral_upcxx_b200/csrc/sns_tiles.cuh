// Tile bodies of the transform and Navier-Stokes passes.
//
// A tile body does the work of one CTA given its tile index `blk`, the CTA's
// thread count and its shared memory.  The single-field kernels (sns_fft.cu,
// sns_ns.cu) call them with blockIdx.x; the ensemble kernels (sns_ens.cu)
// call them for a (box, tile) pair taken from the ensemble's work list, so a
// box advanced inside an ensemble sees the same arithmetic as a box advanced
// alone.  Field pointers come through an accessor (`in(i)`, `out(i)`) so that
// neither caller copies its pointer table to local memory.
#pragma once

#include "sns_fft.cuh"
#include "sns_fft_core.cuh"

namespace sns {

// ---------------------------------------------------------------------------
// Line passes (src/Scalar.cpp:419-566 per axis, src/FFT1D.cpp:95-101 per line)
//
// Thread layout of a tile of W adjacent lines x G groups: thread t owns line
// (w, g) with w = t mod W, and within it positions j + e*TPL (e < E), where
// s = t / W, j = s mod TPL, g = s / TPL.  Consecutive threads hold the same
// position of adjacent lines (unit stride in memory) for W > 1, or adjacent
// positions of one line for W = 1, so the direct global loads and stores are
// coalesced and each thread has E independent loads in flight.  The line FFT
// then starts from registers; shared memory only carries the exchanges
// between radix stages.
struct LineCoord {
  int64_t idx0, step;  // global index of position j, stride between e
  int x, y, z;         // coordinates of position j (3D fields)
};

__device__ __forceinline__ LineCoord line_coord(const LineGeo& geo, int64_t base, int w, int g,
                                                int j, int tpl) {
  LineCoord c;
  c.idx0 = base + w + g * geo.gs + (int64_t)j * geo.ps;
  c.step = (int64_t)tpl * geo.ps;
  c.x = c.y = c.z = 0;
  if (geo.axis >= 0) {
    const int64_t nxy = (int64_t)geo.nx * geo.ny;
    const int64_t z = c.idx0 / nxy;
    const int64_t r = c.idx0 - z * nxy;
    const int64_t y = r / geo.nx;
    c.x = (int)(r - y * geo.nx);
    c.y = (int)y;
    c.z = (int)z;
  }
  return c;
}

// Ask L2 for the 128-byte line holding p (a hint: no register, no wait).
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Prefetch into L2, spread over the CTA's threads, the tile of a line pass
// that starts at element `base` of `src`: G groups (gs apart) of L positions
// (ps apart) of W adjacent elements each; for x lines (ps = 1) the G runs of
// L + W - 1 contiguous elements.  Every address asked for lies inside the
// tile's elements.
template <int L>
__device__ __forceinline__ void prefetch_lines(const char* src, int64_t base, int W, int G,
                                               int64_t gs, int64_t ps, int esz, int nthr) {
  if (ps == 1) {
    const int per_row = ((L - 1 + W) * esz + 127) / 128;
    for (int q = threadIdx.x; q < G * per_row; q += nthr) {
      const int g = q / per_row, c = q - g * per_row;
      prefetch_l2(src + (base + g * gs) * esz + 128 * c);
    }
    return;
  }
  const int per_run = (W * esz + 127) / 128;
  for (int q = threadIdx.x; q < G * L * per_run; q += nthr) {
    const int c = q % per_run, r = q / per_run;
    const int g = r / L, p = r - g * L;
    prefetch_l2(src + (base + g * gs + p * ps) * esz + 128 * c);
  }
}

// K1's tile `bp` (the three components of V) into L2, when it exists.
template <int L, typename C, typename Fields>
__device__ __forceinline__ void prefetch_curl_tile(const LineGeo& geo, const Fields& f,
                                                   int64_t bp) {
  if (geo.pf <= 0 || bp >= geo.TA * geo.TB) return;
  const int64_t basep = (bp % geo.TA) * geo.sa + (bp / geo.TA) * geo.sb;
#pragma unroll
  for (int d = 0; d < 3; d++)
    prefetch_lines<L>(reinterpret_cast<const char*>(f.in(d)), basep, geo.W, geo.G, geo.gs, geo.ps,
                      (int)sizeof(C), (int)blockDim.x);
}

// Element of the thread's line as the prologue forms it.
// PRO_OMEGA: v0..v2 are the z-inverted components of V and d0, d1 the
// z-inverted i kz Vx, i kz Vy (the z derivative taken before the z pass).
template <int PRO, typename C, typename T>
__device__ __forceinline__ C pro_load(const C* __restrict__ src, const C* __restrict__ v0,
                                      const C* __restrict__ v1, const C* __restrict__ v2,
                                      const C* __restrict__ d0, const C* __restrict__ d1,
                                      int field, int64_t idx, T kx, T ky, T kz) {
  if constexpr (PRO == PRO_CURL6) {
    if (field < 3) return src[idx];
    if (field == 3) return csub(ikmul(ky, v2[idx]), ikmul(kz, v1[idx]));
    if (field == 4) return csub(ikmul(kz, v0[idx]), ikmul(kx, v2[idx]));
    return csub(ikmul(kx, v1[idx]), ikmul(ky, v0[idx]));
  } else if constexpr (PRO == PRO_OMEGA) {
    if (field < 3) return src[idx];
    if (field == 3) return csub(ikmul(ky, v2[idx]), d1[idx]);
    if (field == 4) return csub(d0[idx], ikmul(kx, v2[idx]));
    return csub(ikmul(kx, v1[idx]), ikmul(ky, v0[idx]));
  } else {
    return src[idx];
  }
}

// One tile of a line pass: field `blk mod nf`, tile `blk / nf` of `geo`;
// ORD is the radix order of the line FFT (RadixOrder).
template <typename T, int L, int PRO, typename Fields, int ORD = RADIX16_FIRST>
__device__ __forceinline__ void line_pass_tile(const LineGeo& geo, const Fields& f, int nf,
                                               const cx_t<T>* __restrict__ tw, T sg, T scale,
                                               int flags, int wshift, int64_t blk,
                                               cx_t<T>* sm) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;

  const int field = (int)(blk % nf);
  const int64_t t = blk / nf;
  const int64_t base = (t % geo.TA) * geo.sa + (t / geo.TA) * geo.sb;
  const int W = geo.W;
  const int w = threadIdx.x & (W - 1);
  const int s = threadIdx.x >> wshift;
  const int j = s & (TPL - 1);
  const int g = s / TPL;
  const int RS = tile_stride(L, W, (int)sizeof(C));
  C* row = sm + (w + W * g) * RS;
  const LineCoord lc = line_coord(geo, base, w, g, j, TPL);

  C v[E];
  {
    const C* __restrict__ src = reinterpret_cast<const C*>(f.in(field));
    const C* __restrict__ v0 = nullptr;
    const C* __restrict__ v1 = nullptr;
    const C* __restrict__ v2 = nullptr;
    const C* __restrict__ d0 = nullptr;
    const C* __restrict__ d1 = nullptr;
    if constexpr (PRO == PRO_CURL6 || PRO == PRO_OMEGA) {
      v0 = reinterpret_cast<const C*>(f.in(0));
      v1 = reinterpret_cast<const C*>(f.in(1));
      v2 = reinterpret_cast<const C*>(f.in(2));
    }
    if constexpr (PRO == PRO_OMEGA) {
      d0 = reinterpret_cast<const C*>(f.in(3));
      d1 = reinterpret_cast<const C*>(f.in(4));
    }
    // wavenumbers of the line: two are fixed, the one along the axis varies
    const T kx0 = geo.kx_half ? (T)lc.x : (T)freq_i(lc.x, geo.nx),
            ky0 = (T)freq_i(lc.y, geo.ny),
            kz0 = (T)freq_i(lc.z, geo.nz);
    const int naxis = geo.axis == 0 ? geo.nx : geo.axis == 1 ? geo.ny : geo.nz;
    bool ik = false;
    if constexpr (PRO == PRO_IKAXIS) ik = (f.ikmask() >> field) & 1u;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const T kp = (T)freq_i(j + TPL * e, naxis);
      if constexpr (PRO == PRO_IKAXIS) {
        const C x = src[lc.idx0 + e * lc.step];
        v[e] = ik ? ikmul(kp, x) : x;
      } else {
        v[e] = pro_load<PRO, C>(src, v0, v1, v2, d0, d1, field, lc.idx0 + e * lc.step,
                                geo.axis == 0 ? kp : kx0, geo.axis == 1 ? kp : ky0,
                                geo.axis == 2 ? kp : kz0);
      }
    }
  }
  if constexpr (PRO == PRO_LOAD || PRO == PRO_IKAXIS) {
    // with this tile's loads in flight, the tile pf launches ahead into L2
    const int64_t bp = blk + geo.pf;
    if (geo.pf > 0 && bp < geo.TA * geo.TB * nf) {
      const int64_t tp = bp / nf;
      prefetch_lines<L>(reinterpret_cast<const char*>(f.in((int)(bp % nf))),
                        (tp % geo.TA) * geo.sa + (tp / geo.TA) * geo.sb, W, geo.G, geo.gs,
                        geo.ps, (int)sizeof(C), (int)blockDim.x);
    }
  }
  line_fft<L, true, ORD>(v, row, j, tw, sg);

  C* __restrict__ dst = reinterpret_cast<C*>(f.out(field));
  const bool do_scale = flags & PASS_SCALE;
  const bool do_zero = flags & PASS_ZERO_NYQUIST;
  const bool line_on_plane = (geo.axis != 0 && !geo.kx_half && lc.x == (geo.nx >> 1)) ||
                             (geo.axis != 1 && lc.y == (geo.ny >> 1)) ||
                             (geo.axis != 2 && lc.z == (geo.nz >> 1));
  const int half_axis = geo.axis == 0 ? (geo.nx >> 1) : geo.axis == 1 ? (geo.ny >> 1)
                                                                      : (geo.nz >> 1);
#pragma unroll
  for (int e = 0; e < E; e++) {
    C val = v[e];
    if (do_scale) val = cscale(scale, val);
    if (do_zero && (line_on_plane || j + TPL * e == half_axis)) val = mk((T)0, (T)0);
    dst[lc.idx0 + e * lc.step] = val;
  }
}

// One tile of a plain-load line pass (PRO_LOAD) whose input is already in
// shared memory (`stage`, put there by the TMA as one box of field `blk mod
// nf`): position p of line (w, g) at (g L + p) W + w for y lines (the box's
// [z][y][x] order, groups along z) and at (p G + g) W + w for z lines (groups
// along y).  The arithmetic and the epilogue are line_pass_tile's on the same
// values, so both give the same bits.  after_reads() is called by every
// thread once the tile's reads of the stage are issued (the CTA may then
// refill it).
template <typename T, int L, typename Fields, int ORD, typename AfterReads>
__device__ __forceinline__ void line_pass_tile_staged(const LineGeo& geo, const Fields& f, int nf,
                                                      const cx_t<T>* __restrict__ tw, T sg,
                                                      T scale, int flags, int wshift, int64_t blk,
                                                      const cx_t<T>* stage, cx_t<T>* sm,
                                                      AfterReads after_reads) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;
  const int field = (int)(blk % nf);
  const int64_t t = blk / nf;
  const int64_t base = (t % geo.TA) * geo.sa + (t / geo.TA) * geo.sb;
  const int W = geo.W, G = geo.G;
  const int w = threadIdx.x & (W - 1);
  const int s = threadIdx.x >> wshift;
  const int j = s & (TPL - 1);
  const int g = s / TPL;
  const int RS = tile_stride(L, W, (int)sizeof(C));
  C* row = sm + (w + W * g) * RS;
  const LineCoord lc = line_coord(geo, base, w, g, j, TPL);
  // x and y lines: [g][p][w] (x lines have W = 1); z lines: [p][g][w]
  const bool ylines = geo.axis != 2;
  const int q0 = ylines ? (g * L + j) * W + w : (j * G + g) * W + w;
  const int qs = ylines ? TPL * W : TPL * G * W;
  C v[E];
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = stage[q0 + e * qs];
  after_reads();
  line_fft<L, true, ORD>(v, row, j, tw, sg);

  C* __restrict__ dst = reinterpret_cast<C*>(f.out(field));
  const bool do_scale = flags & PASS_SCALE;
  const bool do_zero = flags & PASS_ZERO_NYQUIST;
  const bool line_on_plane = (geo.axis != 0 && !geo.kx_half && lc.x == (geo.nx >> 1)) ||
                             (geo.axis != 1 && lc.y == (geo.ny >> 1)) ||
                             (geo.axis != 2 && lc.z == (geo.nz >> 1));
  const int half_axis = geo.axis == 0 ? (geo.nx >> 1) : geo.axis == 1 ? (geo.ny >> 1)
                                                                      : (geo.nz >> 1);
#pragma unroll
  for (int e = 0; e < E; e++) {
    C val = v[e];
    if (do_scale) val = cscale(scale, val);
    if (do_zero && (line_on_plane || j + TPL * e == half_axis)) val = mk((T)0, (T)0);
    dst[lc.idx0 + e * lc.step] = val;
  }
}

// ---------------------------------------------------------------------------
// K1 of the NS step with one tile for all six outputs: z lines of a W x G tile
// of the three components of V are loaded once (thread layout of
// line_pass_tile, component outermost), the curl omega = i k x V is formed in
// shared memory from the loaded components, and both vectors are
// z-inverse-transformed: out(0..2) = V, out(3..5) = omega.  Shared memory:
// two sets of 3 W G padded rows (V, then omega).
template <typename T, int L, typename Fields>
__device__ __forceinline__ void curl_zpass_tile(const LineGeo& geo, const Fields& f,
                                                const cx_t<T>* __restrict__ tw, int wshift,
                                                int64_t blk, cx_t<T>* sm) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;
  const int W = geo.W, G = geo.G, lines = W * G;
  const int RS = tile_stride(L, W, (int)sizeof(C));
  const int64_t base = (blk % geo.TA) * geo.sa + (blk / geo.TA) * geo.sb;
  prefetch_curl_tile<L, C>(geo, f, blk + geo.pf);
  const int w = threadIdx.x & (W - 1);
  const int s = threadIdx.x >> wshift;
  const int j = s & (TPL - 1);
  const int s2 = s / TPL;
  const int g = s2 % G, d = s2 / G;  // line (w, g) of component d
  const int li = w + W * g;
  C* rowV = sm + (d * lines + li) * RS;
  C* rowW = sm + ((3 + d) * lines + li) * RS;
  const LineCoord lc = line_coord(geo, base, w, g, j, TPL);

  C v[E];
  {
    const C* __restrict__ src = reinterpret_cast<const C*>(
        d == 0 ? f.in(0) : d == 1 ? f.in(1) : f.in(2));
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[lc.idx0 + e * lc.step];
  }
#pragma unroll
  for (int e = 0; e < E; e++) rowV[pad_pos(j + TPL * e)] = v[e];
  __syncthreads();
  {
    // omega_d at this thread's positions from the other two components
    const T kx = geo.kx_half ? (T)lc.x : (T)freq_i(lc.x, geo.nx);
    const T ky = (T)freq_i(lc.y, geo.ny);
    const C* r0 = sm + (0 * lines + li) * RS;
    const C* r1 = sm + (1 * lines + li) * RS;
    const C* r2 = sm + (2 * lines + li) * RS;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int pp = pad_pos(j + TPL * e);
      const T kz = (T)freq_i(j + TPL * e, geo.nz);
      C o;
      if (d == 0)
        o = csub(ikmul(ky, r2[pp]), ikmul(kz, r1[pp]));
      else if (d == 1)
        o = csub(ikmul(kz, r0[pp]), ikmul(kx, r2[pp]));
      else
        o = csub(ikmul(kx, r1[pp]), ikmul(ky, r0[pp]));
      rowW[pp] = o;
    }
  }
  __syncthreads();
  line_fft<L, true>(v, rowV, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? f.out(0) : d == 1 ? f.out(1) : f.out(2));
#pragma unroll
    for (int e = 0; e < E; e++) dst[lc.idx0 + e * lc.step] = v[e];
  }
#pragma unroll
  for (int e = 0; e < E; e++) v[e] = rowW[pad_pos(j + TPL * e)];
  __syncthreads();
  line_fft<L, true>(v, rowW, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? f.out(3) : d == 1 ? f.out(4) : f.out(5));
#pragma unroll
    for (int e = 0; e < E; e++) dst[lc.idx0 + e * lc.step] = v[e];
  }
}

// ---------------------------------------------------------------------------
// K1 with omega formed in registers: each thread z-inverse-transforms its
// component V_d and stores it, then loads the two other components at its
// positions again -- lines the CTA has just read, so the loads are served from
// L1 -- forms omega_d = (i k x V)_d and transforms that.  Shared memory holds
// one set of 3 W G padded rows (the line FFTs' exchanges) and carries no
// component data, so the tile issues 64 shared-memory accesses per thread
// instead of 144.
template <typename T, int L, typename Fields>
__device__ __forceinline__ void curl_zpass_tile_reload(const LineGeo& geo, const Fields& f,
                                                       const cx_t<T>* __restrict__ tw,
                                                       int wshift, int64_t blk, cx_t<T>* sm) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;
  const int W = geo.W, G = geo.G, lines = W * G;
  const int RS = tile_stride(L, W, (int)sizeof(C));
  const int64_t base = (blk % geo.TA) * geo.sa + (blk / geo.TA) * geo.sb;
  prefetch_curl_tile<L, C>(geo, f, blk + geo.pf);
  const int w = threadIdx.x & (W - 1);
  const int s = threadIdx.x >> wshift;
  const int j = s & (TPL - 1);
  const int s2 = s / TPL;
  const int g = s2 % G, d = s2 / G;  // line (w, g) of component d
  C* row = sm + (d * lines + w + W * g) * RS;
  const LineCoord lc = line_coord(geo, base, w, g, j, TPL);
  const C* __restrict__ v0 = reinterpret_cast<const C*>(f.in(0));
  const C* __restrict__ v1 = reinterpret_cast<const C*>(f.in(1));
  const C* __restrict__ v2 = reinterpret_cast<const C*>(f.in(2));
  C v[E];
  {
    const C* __restrict__ src = d == 0 ? v0 : d == 1 ? v1 : v2;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[lc.idx0 + e * lc.step];
  }
  line_fft<L, true>(v, row, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? f.out(0) : d == 1 ? f.out(1) : f.out(2));
#pragma unroll
    for (int e = 0; e < E; e++) dst[lc.idx0 + e * lc.step] = v[e];
  }
  {
    // (ky Vz - kz Vy, kz Vx - kx Vz, kx Vy - ky Vx) times i, as curl_zpass_tile forms it
    const C* __restrict__ pa = d == 0 ? v2 : d == 1 ? v0 : v1;
    const C* __restrict__ pb = d == 0 ? v1 : d == 1 ? v2 : v0;
    const T kx = geo.kx_half ? (T)lc.x : (T)freq_i(lc.x, geo.nx);
    const T ky = (T)freq_i(lc.y, geo.ny);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int64_t q = lc.idx0 + e * lc.step;
      const T kz = (T)freq_i(j + TPL * e, geo.nz);
      const C a = pa[q], b = pb[q];
      if (d == 0)
        v[e] = csub(ikmul(ky, a), ikmul(kz, b));
      else if (d == 1)
        v[e] = csub(ikmul(kz, a), ikmul(kx, b));
      else
        v[e] = csub(ikmul(kx, a), ikmul(ky, b));
    }
  }
  // the last stage of the first transform read the row before a block barrier,
  // so the second may write it at once
  line_fft<L, true>(v, row, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? f.out(3) : d == 1 ? f.out(4) : f.out(5));
#pragma unroll
    for (int e = 0; e < E; e++) dst[lc.idx0 + e * lc.step] = v[e];
  }
}

// K1 from a staged tile: the three components of V for the tile are already
// in shared memory (`stage`, put there by the TMA): component c, position p
// of line (w, g) at c L W G + (p G + g) W + w, the [z][y][x] order of the
// TMA box.  The arithmetic is curl_zpass_tile_reload's with its loads of V
// read from the stage, so both give the same bits.  after_reads() is called
// by every thread once the tile's last read of the stage is issued (the CTA
// may then refill the stage).
template <typename T, int L, typename Fields, typename AfterReads>
__device__ __forceinline__ void curl_zpass_tile_staged(const LineGeo& geo, const Fields& f,
                                                       const cx_t<T>* __restrict__ tw,
                                                       int wshift, int64_t blk,
                                                       const cx_t<T>* stage, cx_t<T>* sm,
                                                       AfterReads after_reads) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;
  const int W = geo.W, G = geo.G, lines = W * G;
  const int RS = tile_stride(L, W, (int)sizeof(C));
  const int64_t base = (blk % geo.TA) * geo.sa + (blk / geo.TA) * geo.sb;
  const int w = threadIdx.x & (W - 1);
  const int s = threadIdx.x >> wshift;
  const int j = s & (TPL - 1);
  const int s2 = s / TPL;
  const int g = s2 % G, d = s2 / G;  // line (w, g) of component d
  C* row = sm + (d * lines + w + W * g) * RS;
  const LineCoord lc = line_coord(geo, base, w, g, j, TPL);
  const int q0 = j * lines + g * W + w, qs = TPL * lines, comp = L * lines;
  C v[E];
  {
    const C* sv = stage + d * comp;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = sv[q0 + e * qs];
  }
  line_fft<L, true>(v, row, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? f.out(0) : d == 1 ? f.out(1) : f.out(2));
#pragma unroll
    for (int e = 0; e < E; e++) dst[lc.idx0 + e * lc.step] = v[e];
  }
  {
    // (ky Vz - kz Vy, kz Vx - kx Vz, kx Vy - ky Vx) times i, as curl_zpass_tile forms it
    const C* pa = stage + (d == 0 ? 2 : d == 1 ? 0 : 1) * comp;
    const C* pb = stage + (d == 0 ? 1 : d == 1 ? 2 : 0) * comp;
    const T kx = geo.kx_half ? (T)lc.x : (T)freq_i(lc.x, geo.nx);
    const T ky = (T)freq_i(lc.y, geo.ny);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int q = q0 + e * qs;
      const T kz = (T)freq_i(j + TPL * e, geo.nz);
      const C a = pa[q], b = pb[q];
      if (d == 0)
        v[e] = csub(ikmul(ky, a), ikmul(kz, b));
      else if (d == 1)
        v[e] = csub(ikmul(kz, a), ikmul(kx, b));
      else
        v[e] = csub(ikmul(kx, a), ikmul(ky, b));
    }
  }
  after_reads();
  line_fft<L, true>(v, row, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? f.out(3) : d == 1 ? f.out(4) : f.out(5));
#pragma unroll
    for (int e = 0; e < E; e++) dst[lc.idx0 + e * lc.step] = v[e];
  }
}

// ---------------------------------------------------------------------------
// K3 of the NS step: x lines -- inverse 6 fields, 1/N^2-scaled complex cross
// product u x omega, forward 3 fields (src/Vector.cpp:79-89).  A tile is G
// rows of all six fields; f.in(0..5) = (u, omega), f.out(0..2) = the product.
//
// The tile's input comes through load(fld, gl, j, v): the E elements j + e*TPL
// of row gl of field fld (xcross_tile reads them from HBM; the TMA-staged pass
// from the shared-memory stage).
template <typename T, int L, typename Fields, typename Load>
__device__ __forceinline__ void xcross_tile_from(const Fields& f, const cx_t<T>* __restrict__ tw,
                                                 int G, T scale2, int64_t blk, int nthr,
                                                 cx_t<T>* sm, Load load) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL, RS = xrow_stride(L, (int)sizeof(C));
  const int64_t row0 = blk * G;
  const int per = G * L;

  // thread t owns line t / TPL (field-major: field = line / G, row = line % G)
  // at positions j + e*TPL, E elements in registers
  const int j = threadIdx.x % TPL, line = threadIdx.x / TPL;
  const int fld = line / G, gl = line - fld * G;
  C* row = sm + line * RS;
  C v[E];
  load(fld, gl, j, v);
  line_fft<L>(v, row, j, tw, (T)1);
#pragma unroll
  for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
  __syncthreads();

  // c = (u/N) x (omega/N): u in rows of fields 0..2, omega in 3..5
  for (int q = threadIdx.x; q < per; q += nthr) {
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
    C* __restrict__ dst = reinterpret_cast<C*>(f.out(fld));
    const int64_t i0 = (row0 + gl) * L + j;
#pragma unroll
    for (int e = 0; e < E; e++) dst[i0 + TPL * e] = v[e];
  }
}

// K3 tile with its loads from HBM straight into registers (E per thread in
// flight), optionally asking L2 for the rows of tile blk + pf first.
template <typename T, int L, typename Fields>
__device__ __forceinline__ void xcross_tile(const Fields& f, const cx_t<T>* __restrict__ tw, int G,
                                            T scale2, int64_t blk, int nthr, cx_t<T>* sm,
                                            int64_t pf = 0, int64_t nblk = 0) {
  using C = cx_t<T>;
  constexpr int E = LinePlan<L>::E, TPL = LinePlan<L>::TPL;
  xcross_tile_from<T, L>(f, tw, G, scale2, blk, nthr, sm, [&](int fld, int gl, int j, C (&v)[E]) {
    const C* __restrict__ src = reinterpret_cast<const C*>(f.in(fld));
    const int64_t i0 = (blk * G + gl) * L + j;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[i0 + TPL * e];
    if (pf > 0 && blk + pf < nblk) {
      // with this tile's loads in flight, the six input rows of tile blk + pf
      // into L2
#pragma unroll
      for (int fl = 0; fl < 6; fl++)
        prefetch_lines<L>(reinterpret_cast<const char*>(f.in(fl)), (blk + pf) * G * L, 1, G, L, 1,
                          (int)sizeof(C), nthr);
    }
  });
}

// ---------------------------------------------------------------------------
// K5 of the NS step: z lines -- forward 3 fields + Nyquist zeroing, then the
// AB2 / projection / CN update per mode (ns.cpp:170-187) and the FP64
// diagnostics of the new velocity (ns.cpp:206-210).
struct UpdateArgs {
  const void* U[3];  // cross1 after x, y forward passes
  void* V[3];        // in: V1, out: V (new)
  void* C0[3];       // in: cross0, out: cross1
  int nx, ny, nz;
  int lx;         // log2(nx)
  int W;          // adjacent z lines per tile (may exceed nx: rows of the xy plane)
  double hK;      // K/2
  double nuhK;    // nu*K/2
  double* stats;  // per tile: sum|div|, sum|V|^2, sum|k x V|^2, max|div|
  // SGS: eddy stress tau_xx, tau_yy, tau_zz, tau_xy, tau_xz, tau_yz after the
  // x and y forward passes; z-transformed in the tile, its divergence
  // i k_j tau_ij joins cross1 before the Nyquist zeroing
  const void* tau[6];
  double kc2;  // spectral cutoff |k|^2 <= kc2 of an LES run (1e300: none)
  int kx_half;  // half-spectrum fields (see LineGeo::kx_half)
  // SGS: the stress divergence is weighted by clamp((|k| - sgs_klo) sgs_kinv, 0, 1)
  double sgs_klo, sgs_kinv;
  // L2 prefetch distance in tiles (0: none)
  int64_t pf;
  // the carried z-inverse pass (zfwd_update_curl_tile): out(0..2) = the new
  // V, out(3..5) = i k x V, both z-inverse-transformed
  void* Uo[6];
  // ask L2 for this tile's V and C0 before its z-forward (0: no)
  int pf_self;
};

// Field f of the update's z-forward: the cross product (f < 3) or, with the
// eddy stress, tau_{f-3}; selected with constant indices.
__device__ __forceinline__ const void* update_field(const UpdateArgs& a, int f) {
  const void* r = a.U[0];
  if (f == 1) r = a.U[1];
  if (f == 2) r = a.U[2];
#pragma unroll
  for (int q = 0; q < 6; q++)
    if (f == 3 + q) r = a.tau[q];
  return r;
}

// Tile `blk` holds the W z lines whose xy-plane offsets are blk*W .. blk*W+W-1.
// With SGS the six stress fields are z-transformed in the same tile (9 fields
// in shared memory, 9 W TPL threads).
//
// The z lines come through load(fld, w, j, v): the E elements j + e*TPL of
// line w of field fld (zfwd_update_tile reads them from HBM; the TMA-staged
// pass from its shared-memory stage).
//
// KEEP = true also leaves the new velocity in the tile's first three rows
// (component d of line w at (d W + w) RS + pad_pos(z), where the z-forward of
// the cross product was), ordered before the caller's reads by the block
// barrier of the diagnostics' reduction.
template <typename T, int L, bool SGS, bool KEEP = false, typename Load>
__device__ __forceinline__ void zfwd_update_tile_from(const UpdateArgs& a,
                                                      const cx_t<T>* __restrict__ tw, int64_t blk,
                                                      int nthr, cx_t<T>* sm, double (*red)[32],
                                                      Load load) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL;

  const int W = a.W;
  const int RS = tile_stride(L, W, (int)sizeof(C));
  const int64_t nxy = (int64_t)a.nx * a.ny;
  const int64_t base = blk * W;
  const int per = W * L;

  // thread t owns z line (field, base + w) at positions j + e*TPL with
  // w = t mod W, j = (t / W) mod TPL, field = t / (W*TPL): consecutive threads
  // load adjacent x, so the direct loads are coalesced.  A CTA of half the
  // threads (nthr = NF W TPL / 2, W even) transforms the tile in two halves of
  // W/2 adjacent lines, one after the other: a wide tile (W = 32) keeps the
  // update's rows of 32 adjacent x within the thread limit.
  {
    constexpr int NF = SGS ? 9 : 3;
    const int WH = NF * W * TPL > nthr ? W / 2 : W;  // lines along x per half
#pragma unroll 1
    for (int w0 = 0; w0 < W; w0 += WH) {
      const int w = w0 + threadIdx.x % WH, s = threadIdx.x / WH;
      const int j = s % TPL, fld = s / TPL;
      C* row = sm + (fld * W + w) * RS;
      C v[E];
      load(fld, w, j, v);
      line_fft<L, true>(v, row, j, tw, (T)-1);
#pragma unroll
      for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
    }
  }
  __syncthreads();

  const T hK = (T)a.hK, nuhK = (T)a.nuhK;
  double s_div = 0, s_e = 0, s_w = 0, m_div = 0;
  C* __restrict__ Vp[3] = {reinterpret_cast<C*>(a.V[0]), reinterpret_cast<C*>(a.V[1]),
                           reinterpret_cast<C*>(a.V[2])};
  C* __restrict__ Cp[3] = {reinterpret_cast<C*>(a.C0[0]), reinterpret_cast<C*>(a.C0[1]),
                           reinterpret_cast<C*>(a.C0[2])};
  auto update_point = [&](int q, const C (&V1)[3], const C (&c0)[3]) {
    const int w = q % W, z = q / W;
    const int64_t xy = base + w;
    const int x = (int)(xy & (a.nx - 1)), y = (int)(xy >> a.lx);
    const int64_t idx = xy + nxy * z;
    const T kx = a.kx_half ? (T)x : (T)freq_i(x, a.nx);
    const T ky = (T)freq_i(y, a.ny), kz = (T)freq_i(z, a.nz);
    const double k2d = (double)kx * kx + (double)ky * ky + (double)kz * kz;
    // modes beyond the cutoff are not evolved (zero velocity and history)
    const bool cut = k2d > a.kc2;
    const bool nyq = cut || y == (a.ny >> 1) || (!a.kx_half && x == (a.nx >> 1)) ||
                     z == (a.nz >> 1);
    // half spectrum: each stored kx > 0 mode stands for itself and its conjugate
    const double wgt = (a.kx_half && x > 0) ? 2.0 : 1.0;
    C c1[3];
#pragma unroll
    for (int d = 0; d < 3; d++) c1[d] = nyq ? mk((T)0, (T)0) : sm[(d * W + w) * RS + pad_pos(z)];
    if constexpr (SGS) {
      const T ws = (T)fmin(1.0, fmax(0.0, (sqrt(k2d) - a.sgs_klo) * a.sgs_kinv));
      if (!nyq && ws > (T)0) {
        C t6[6];
#pragma unroll
        for (int q = 0; q < 6; q++) t6[q] = sm[((3 + q) * W + w) * RS + pad_pos(z)];
        // (div tau)_i = i (kx tau_ix + ky tau_iy + kz tau_iz)
        const C f0 = cadd(cadd(ikmul(kx, t6[0]), ikmul(ky, t6[3])), ikmul(kz, t6[4]));
        const C f1 = cadd(cadd(ikmul(kx, t6[3]), ikmul(ky, t6[1])), ikmul(kz, t6[5]));
        const C f2 = cadd(cadd(ikmul(kx, t6[4]), ikmul(ky, t6[5])), ikmul(kz, t6[2]));
        c1[0] = cadd(c1[0], cscale(ws, f0));
        c1[1] = cadd(c1[1], cscale(ws, f1));
        c1[2] = cadd(c1[2], cscale(ws, f2));
      }
    }
    const T kk[3] = {kx, ky, kz};
    const T k2 = kx * kx + ky * ky + kz * kz;
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
      if (cut) vv = mk((T)0, (T)0);
      Vn[d] = vv;
      Vp[d][idx] = vv;
      Cp[d][idx] = c1[d];
      if constexpr (KEEP) sm[(d * W + w) * RS + pad_pos(z)] = vv;
    }
    // diagnostics of the new velocity: per-mode terms in T, sums in FP64
    const C dv = cadd(cadd(ikmul(kx, Vn[0]), ikmul(ky, Vn[1])), ikmul(kz, Vn[2]));
    const double ad = (double)sqrt(dv.x * dv.x + dv.y * dv.y);
    s_div += wgt * ad;
    m_div = fmax(m_div, ad);
    T e2 = 0;
#pragma unroll
    for (int d = 0; d < 3; d++) e2 += Vn[d].x * Vn[d].x + Vn[d].y * Vn[d].y;
    const C om0 = csub(ikmul(ky, Vn[2]), ikmul(kz, Vn[1]));
    const C om1 = csub(ikmul(kz, Vn[0]), ikmul(kx, Vn[2]));
    const C om2 = csub(ikmul(kx, Vn[1]), ikmul(ky, Vn[0]));
    const T w2 = om0.x * om0.x + om0.y * om0.y + om1.x * om1.x + om1.y * om1.y +
                 om2.x * om2.x + om2.y * om2.y;
    s_e += wgt * (double)e2;
    s_w += wgt * (double)w2;
  };
  // two points per iteration: the 12 global loads of both are issued first
  for (int q0 = threadIdx.x; q0 < per; q0 += 2 * nthr) {
    const int q1 = q0 + nthr;
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
  const int warp = threadIdx.x >> 5, nwarps = (nthr + 31) >> 5;
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
    double* out = a.stats + 4 * blk;
    out[0] = t0;
    out[1] = t1;
    out[2] = t2;
    out[3] = t3;
  }
}

// K5 tile with its loads from HBM straight into registers, optionally asking
// L2 for the inputs of tile blk + pf first.
template <typename T, int L, bool SGS = false, bool KEEP = false>
__device__ __forceinline__ void zfwd_update_tile(const UpdateArgs& a,
                                                 const cx_t<T>* __restrict__ tw, int64_t blk,
                                                 int nthr, cx_t<T>* sm, double (*red)[32]) {
  using C = cx_t<T>;
  constexpr int E = LinePlan<L>::E, TPL = LinePlan<L>::TPL;
  const int W = a.W;
  const int64_t nxy = (int64_t)a.nx * a.ny;
  const int64_t base = blk * W;
  zfwd_update_tile_from<T, L, SGS, KEEP>(a, tw, blk, nthr, sm, red, [&](int fld, int w, int j, C (&v)[E]) {
    const C* __restrict__ src = reinterpret_cast<const C*>(
        SGS ? update_field(a, fld) : (fld == 0 ? a.U[0] : fld == 1 ? a.U[1] : a.U[2]));
    const int64_t i0 = base + w + nxy * j;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[i0 + nxy * (TPL * e)];
    if (!SGS && a.pf_self) {
      // with the cross product's loads in flight, ask L2 for this tile's V
      // and C0, so that the update's loads after the z-forward find them there
#pragma unroll
      for (int d = 0; d < 3; d++) {
        prefetch_lines<L>(reinterpret_cast<const char*>(a.V[d]), base, W, 1, 0, nxy,
                          (int)sizeof(C), nthr);
        prefetch_lines<L>(reinterpret_cast<const char*>(a.C0[d]), base, W, 1, 0, nxy,
                          (int)sizeof(C), nthr);
      }
    }
    if (!SGS && a.pf > 0 && (blk + a.pf) * W < nxy) {
      // and tile blk + pf's cross product, V and C0
      const int64_t bp = (blk + a.pf) * W;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        prefetch_lines<L>(reinterpret_cast<const char*>(a.U[d]), bp, W, 1, 0, nxy,
                          (int)sizeof(C), nthr);
        prefetch_lines<L>(reinterpret_cast<const char*>(a.V[d]), bp, W, 1, 0, nxy,
                          (int)sizeof(C), nthr);
        prefetch_lines<L>(reinterpret_cast<const char*>(a.C0[d]), bp, W, 1, 0, nxy,
                          (int)sizeof(C), nthr);
      }
    }
  });
}

// K5 with the next step's K1 carried in it: the update of zfwd_update_tile,
// then the z-inverse of the new velocity and of its curl omega = i k x V from
// the tile's rows (KEEP), into a.Uo -- what K1 of the next step would compute
// from V in HBM, with the arithmetic of curl_zpass_tile_staged (same line FFT,
// same products), so a step that starts from these fields skips K1 and the
// re-read of V.  The tile's W z lines all lie in one xy-plane run, so their
// (kx, ky) come from the line's xy offset.  Shared memory: the 3 W rows of the
// update, then 3 W exchange rows for the line FFTs (the rows of V stay intact
// while the curl reads them).
//
// RELOAD = true keeps K5's shared memory (3 W rows, so as many CTAs per SM
// as K5): the new velocity is read back from V, which this CTA has just
// written (L1/L2, not DRAM; the block barrier of the diagnostics makes the
// stores visible), and each thread's own row serves as its exchange row, as
// in curl_zpass_tile_reload.
template <typename T, int L, bool RELOAD = false>
__device__ __forceinline__ void zfwd_update_curl_tile(const UpdateArgs& a,
                                                      const cx_t<T>* __restrict__ tw, int64_t blk,
                                                      int nthr, cx_t<T>* sm, double (*red)[32]) {
  using C = cx_t<T>;
  constexpr int E = LinePlan<L>::E, TPL = LinePlan<L>::TPL;
  zfwd_update_tile<T, L, false, !RELOAD>(a, tw, blk, nthr, sm, red);
  const int W = a.W;
  const int RS = tile_stride(L, W, (int)sizeof(C));
  const int64_t nxy = (int64_t)a.nx * a.ny;
  const int w = threadIdx.x % W, s = threadIdx.x / W;
  const int j = s % TPL, d = s / TPL;  // line w of component d, positions j + e TPL
  const int64_t xy = blk * W + w;
  const int x = (int)(xy & (a.nx - 1)), y = (int)(xy >> a.lx);
  const int64_t idx0 = xy + nxy * j, step = nxy * TPL;
  const C* v0 = reinterpret_cast<const C*>(a.V[0]);
  const C* v1 = reinterpret_cast<const C*>(a.V[1]);
  const C* v2 = reinterpret_cast<const C*>(a.V[2]);
  const C* vr = sm + (d * W + w) * RS;
  C* xrow = RELOAD ? sm + (d * W + w) * RS : sm + (3 * W + d * W + w) * RS;
  C v[E];
  if constexpr (RELOAD) {
    const C* src = d == 0 ? v0 : d == 1 ? v1 : v2;
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[idx0 + e * step];
  } else {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = vr[pad_pos(j + TPL * e)];
  }
  line_fft<L, true>(v, xrow, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? a.Uo[0] : d == 1 ? a.Uo[1] : a.Uo[2]);
#pragma unroll
    for (int e = 0; e < E; e++) dst[idx0 + e * step] = v[e];
  }
  {
    // (ky Vz - kz Vy, kz Vx - kx Vz, kx Vy - ky Vx) times i, as curl_zpass_tile forms it
    const C* pa = sm + ((d == 0 ? 2 : d == 1 ? 0 : 1) * W + w) * RS;
    const C* pb = sm + ((d == 0 ? 1 : d == 1 ? 2 : 0) * W + w) * RS;
    const C* ga = d == 0 ? v2 : d == 1 ? v0 : v1;
    const C* gb = d == 0 ? v1 : d == 1 ? v2 : v0;
    const T kx = a.kx_half ? (T)x : (T)freq_i(x, a.nx);
    const T ky = (T)freq_i(y, a.ny);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int p = j + TPL * e;
      const T kz = (T)freq_i(p, a.nz);
      const C va = RELOAD ? ga[idx0 + e * step] : pa[pad_pos(p)];
      const C vb = RELOAD ? gb[idx0 + e * step] : pb[pad_pos(p)];
      if (d == 0)
        v[e] = csub(ikmul(ky, va), ikmul(kz, vb));
      else if (d == 1)
        v[e] = csub(ikmul(kz, va), ikmul(kx, vb));
      else
        v[e] = csub(ikmul(kx, va), ikmul(ky, vb));
    }
  }
  // the last stage of the first transform read its exchange row before a
  // block barrier, so the second may write it at once
  line_fft<L, true>(v, xrow, j, tw, (T)1);
  {
    C* __restrict__ dst = reinterpret_cast<C*>(d == 0 ? a.Uo[3] : d == 1 ? a.Uo[4] : a.Uo[5]);
#pragma unroll
    for (int e = 0; e < E; e++) dst[idx0 + e * step] = v[e];
  }
}

// Entry i of a pointer table in kernel parameters, selected with constant
// indices so that the table is read in place rather than copied to local
// memory for a dynamic index.
__device__ __forceinline__ void* select_ptr(void* const (&a)[kMaxFields], int i) {
  void* r = a[0];
#pragma unroll
  for (int k = 1; k < kMaxFields; k++)
    if (i == k) r = a[k];
  return r;
}

// Field accessor over a FieldPtrs held in kernel parameters.
struct ParamFields {
  const FieldPtrs& f;
  __device__ __forceinline__ const void* in(int i) const { return select_ptr(f.in, i); }
  __device__ __forceinline__ void* out(int i) const { return select_ptr(f.out, i); }
  __device__ __forceinline__ unsigned ikmask() const { return f.ikmask; }
};

}  // namespace sns
