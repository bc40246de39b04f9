// Register/shared-memory FFT core for one line of compile-time length L.
//
// Each line is owned by TPL = L/E threads that hold E elements each in
// registers (E = 16 for L >= 16).  Stages follow the Stockham formulation of
// Govindaraju et al., "High Performance Discrete Fourier Transforms on Graphics
// Processors" (SC'08): a radix-R stage with Ns outputs already combined reads
// x[jb + r*L/R], twiddles by W_{Ns R}^{(jb mod Ns) r}, runs an R-point DFT and
// writes y[(jb/Ns)*Ns*R + jb mod Ns + r*Ns].  Thread j of a line runs the
// butterflies jb = j + m*TPL, so at every stage boundary it holds elements
// j + TPL*e -- the natural-order layout the caller loads and stores.  Stages
// exchange data through one padded shared-memory row per line.
//
// Twiddles come from a table tw[m] = exp(-2 pi i m / L) generated in FP64 on
// the host and rounded to T; the inverse direction conjugates on the fly.
#pragma once

#include "sns_common.cuh"

namespace sns {

// Padded shared-memory index of line position p: one spare slot per 16
// elements keeps the strided stage writes off a single bank.
__host__ __device__ constexpr int pad_pos(int p) { return p + (p >> 4); }
// Row stride of a line in shared memory, odd so that the column-wise tile
// loads of strided axes hit distinct banks.
__host__ __device__ constexpr int row_stride(int L) {
  return (pad_pos(L) & 1) ? pad_pos(L) : pad_pos(L) + 1;
}
// Row stride of a tile whose accesses are served per group of P = 128 / esz
// lanes (a half-warp for 8-byte elements, a quarter-warp for 16-byte ones):
// such a group holds P / J lines of J = min(TPL, P / W) consecutive positions
// for runs of W adjacent lines (thread index w fastest; W = 1 for single x
// lines), so its P lanes fall on distinct element slots (modulo P) when the
// stride is J times an odd number.  J = 1 is an odd stride.
__host__ __device__ constexpr int tile_stride(int L, int W, int esz = 8) {
  const int P = 128 / esz;
  const int tpl = L >= 16 ? L / 16 : 1;
  const int J = W >= P ? 1 : (P / W < tpl ? P / W : tpl);
  int rs = pad_pos(L);
  if (J >= P) return rs;
  while (rs % J != 0 || ((rs / J) & 1) == 0) rs++;
  return rs;
}
// Tiles of x lines.
__host__ __device__ constexpr int xrow_stride(int L, int esz = 8) { return tile_stride(L, 1, esz); }

// Radix orders of a line (all give the same transform to rounding; the
// autotuner picks one per line length):
//   RADIX16_FIRST  radix-16 stages, the remainder (2, 4 or 8) last
//   RADIX_REM_FIRST  the remainder first, then the radix-16 stages
//   RADIX8  radix-8 stages, the remainder (2 or 4) last
enum RadixOrder : int { RADIX16_FIRST = 0, RADIX_REM_FIRST = 1, RADIX8 = 2, kRadixOrders = 3 };

template <int L, int ORD = RADIX16_FIRST>
struct LinePlan {
  static constexpr int E = (L >= 16) ? 16 : L;  // elements per thread
  static constexpr int TPL = L / E;             // threads per line
  static constexpr int BIG = (ORD == RADIX8 && L >= 8) ? 8 : 16;  // the repeated radix
  static constexpr int REM = [] {
    int r = L;
    while (r >= BIG && r % BIG == 0) r /= BIG;
    return r;
  }();
  static constexpr int NBIG = [] {
    int c = 0, r = L;
    while (r >= BIG && r % BIG == 0) { r /= BIG; c++; }
    return c;
  }();
  static constexpr int NSTAGE = NBIG + (REM > 1 ? 1 : 0);
  // radix of stage s
  __host__ __device__ static constexpr int radix(int s) {
    if (ORD == RADIX_REM_FIRST && REM > 1) return s == 0 ? REM : BIG;
    return s < NBIG ? BIG : REM;
  }
  static_assert(L >= 2 && (L & (L - 1)) == 0, "power-of-two line length");
  static_assert(E % BIG == 0 || L < BIG, "a thread holds whole butterflies");
};

// W_R^k for R in {8, 16}: cos and sin(2 pi k / 16) for k = 0..15.
__device__ __forceinline__ double tw16_c(int k) {
  constexpr double c[16] = {1.0,
                            0.92387953251128675613,
                            0.70710678118654752440,
                            0.38268343236508977173,
                            0.0,
                            -0.38268343236508977173,
                            -0.70710678118654752440,
                            -0.92387953251128675613,
                            -1.0,
                            -0.92387953251128675613,
                            -0.70710678118654752440,
                            -0.38268343236508977173,
                            0.0,
                            0.38268343236508977173,
                            0.70710678118654752440,
                            0.92387953251128675613};
  return c[k & 15];
}
__device__ __forceinline__ double tw16_s(int k) { return tw16_c((k + 12) & 15); }

// In-register DFT of size R: a[s] <- sum_q W_R^{qs} a[q], W_R = exp(sg*2 pi i/R).
template <int R, typename C, typename T>
__device__ __forceinline__ void dft(C* a, T sg) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2) {
    C t = a[1];
    a[1] = csub(a[0], t);
    a[0] = cadd(a[0], t);
  } else if constexpr (R == 4) {
    C t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
    C t2 = cadd(a[1], a[3]), d = csub(a[1], a[3]);
    C t3 = mk(-sg * d.y, sg * d.x);  // d * (sg i)
    a[0] = cadd(t0, t2);
    a[2] = csub(t0, t2);
    a[1] = cadd(t1, t3);
    a[3] = csub(t1, t3);
  } else {
    // radix-2 decimation in time: R = 2 * (R/2)
    constexpr int H = R / 2;
    C e[H], o[H];
#pragma unroll
    for (int i = 0; i < H; i++) {
      e[i] = a[2 * i];
      o[i] = a[2 * i + 1];
    }
    dft<H>(e, sg);
    dft<H>(o, sg);
#pragma unroll
    for (int k = 0; k < H; k++) {
      C t;
      if (k == 0) {
        t = o[0];
      } else if (2 * k == H) {
        t = mk(-sg * o[k].y, sg * o[k].x);  // W_R^{R/4} = sg i
      } else {
        constexpr int step = 16 / R;
        const T c = (T)tw16_c(k * step), s = sg * (T)tw16_s(k * step);
        t = mk(o[k].x * c - o[k].y * s, o[k].x * s + o[k].y * c);
      }
      a[k] = cadd(e[k], t);
      a[k + H] = csub(e[k], t);
    }
  }
}

// Synchronise the threads that share a line.  Lines of up to 32 threads sit
// inside one warp (thread index = j + TPL*line), wider lines span the block.
template <int TPL>
__device__ __forceinline__ void line_sync() {
  if constexpr (TPL <= 32)
    __syncwarp();
  else
    __syncthreads();
}

// Transform one line in place.  On entry v[e] holds element j + TPL*e of the
// line, on exit the transformed element with the same index.  Line position p
// lives at base[idx(p)] in shared memory; `tw` is the length-L forward
// twiddle table, sg = -1 forward, +1 inverse; `sync()` synchronises the
// threads that share the line.  The first stage writes the line's slots at
// once, so the caller synchronises the line after its own reads of them.
template <int L, int ORD = RADIX16_FIRST, typename C, typename T, typename Idx, typename Sync>
__device__ __forceinline__ void line_fft_at(C (&v)[LinePlan<L>::E], C* base, Idx idx, int j,
                                            const C* __restrict__ tw, T sg, Sync sync) {
  using P = LinePlan<L, ORD>;
  constexpr int E = P::E, TPL = P::TPL;
  int Ns = 1;
#pragma unroll
  for (int s = 0; s < P::NSTAGE; s++) {
    const int R = P::radix(s);
    const bool last = (s == P::NSTAGE - 1);
    if (s > 0) {
#pragma unroll
      for (int e = 0; e < E; e++) v[e] = base[idx(j + TPL * e)];
      sync();
    }
    // butterflies m = 0 .. E/R-1 of this thread
#pragma unroll
    for (int m = 0; m < 16; m++) {
      if (m >= E / R) break;
      const int jb = j + m * TPL;
      C a[16];
#pragma unroll
      for (int r = 0; r < 16; r++)
        if (r < R) a[r] = v[m + (E / R) * r];
      if (s > 0) {
        const int k = jb % Ns;
        const int step = L / (Ns * R);
#pragma unroll
        for (int r = 1; r < 16; r++) {
          if (r < R) {
            C w = tw[(k * r * step) & (L - 1)];
            w.y *= -sg;  // the table holds exp(-i..); sg = +1 conjugates it
            a[r] = cmul(a[r], w);
          }
        }
      }
      switch (R) {
        case 2: dft<2>(a, sg); break;
        case 4: dft<4>(a, sg); break;
        case 8: dft<8>(a, sg); break;
        default: dft<16>(a, sg); break;
      }
      if (last) {
#pragma unroll
        for (int r = 0; r < 16; r++)
          if (r < R) v[m + (E / R) * r] = a[r];
      } else {
        const int b = (jb / Ns) * Ns * R + (jb % Ns);
#pragma unroll
        for (int r = 0; r < 16; r++)
          if (r < R) base[idx(b + r * Ns)] = a[r];
      }
    }
    if (!last) sync();
    Ns *= R;
  }
}

// line_fft_at on a padded row: position p at row[pad_pos(p)].  Every thread of
// the block must call this (it may synchronise the block when TPL > 32).
// BLOCK = true synchronises the whole block between stages, for layouts in
// which the threads of a line are not confined to one warp.
template <int L, bool BLOCK = false, int ORD = RADIX16_FIRST, typename C, typename T>
__device__ __forceinline__ void line_fft(C (&v)[LinePlan<L>::E], C* row, int j,
                                         const C* __restrict__ tw, T sg) {
  line_fft_at<L, ORD>(
      v, row, [](int p) { return pad_pos(p); }, j, tw, sg, [] {
        if constexpr (BLOCK)
          __syncthreads();
        else
          line_sync<LinePlan<L>::TPL>();
      });
}

}  // namespace sns
