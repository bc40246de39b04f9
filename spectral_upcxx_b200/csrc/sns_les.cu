// Eddy-viscosity closure of the fused NS step, and the data kernels of the
// learned closure (spectral filter, SGS targets, energy spectrum).
//
// No reference counterpart: exec/ns.cpp has no subgrid model.  The closure
// step adds the divergence of the eddy stress tau_ij = 2 nu_t S_ij to the
// nonlinear term cross1 (ns.cpp:203-206) and is otherwise the ns.cpp step:
//
//   z-inverse of V and of d_z V = i k_z V (derivative on the way in)   6 out
//   y-inverse of those and of d_y V (i k_y times the z-inverted V)     9 out
//   x-inverse of the 9 and of d_x V (i k_x times the y-inverted V),
//   closure (nu_t by Smagorinsky or the MLP on the tensor cores, u x omega
//   and tau_ij per point), x-forward of the 9 results: one fused pass
//   (k_x, k_y are constant along z lines and k_x along y lines, so each
//   derivative is transformed only from the pass of its own axis on)
//   y-forward of u x omega, tau             1 x 9
//   z-forward of u x omega and tau, + i k_j tau_ij, then the AB2 /
//   projection / CN update                  1 x 9 in, 6 out
#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>
#include <type_traits>
#include <string>

#include "../../include/spectral_b200.h"
#include "sns_ens.cuh"
#include "sns_fft.cuh"
#include "sns_les.cuh"
#include "sns_mlp.cuh"
#include "sns_tc.cuh"
#include "sns_ops.cuh"
#include "sns_tiles.cuh"

namespace sns {

// Rows of x lines per CTA of the fused x pass: 12 fields x G rows x TPL
// threads = 384 whatever the line length (TPL = L / 16).
constexpr int kXlesThreads = 384;

// The MLP of the x pass on tcgen05: the CTA's 512 points as four tiles of
// 128, run by warps 0-3 (thread m owns point m of the tile): features into the
// K-major A tile, layer 1 (one MMA, b1 through the bias columns), ReLU/BF16
// epilogue into the layer-2 A tile, layer 2 (four MMAs + the b2 slice), output
// epilogue; 64 tensor-memory columns per CTA, bounded mbarrier waits.
struct __align__(128) XlesTcSmem {
  unsigned char W1[kMlpHidden * kMlpK1 * 2];
  unsigned char W2[kMlpHidden * kMlpHidden * 2];
  unsigned char B2[kMlpHidden * 16 * 2];
  unsigned char ONES[128 * 16 * 2];
  unsigned char X[128 * kMlpK1 * 2];
  unsigned char H[128 * kMlpHidden * 2];
  float w3[kMlpHidden];
  float b3, s_in, s_out;
  uint64_t mbar;
  uint32_t tmem;
  int abort;
};
struct XlesNoSmem {};

__device__ int g_xles_tc_status;  // nonzero: a tensor-core wait of k_xles ran out

__device__ __forceinline__ void mlp_warps_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

struct XlesArgs {
  FieldPtrs f;  // in: u (3), A_ij = d_j u_i (9) after the z and y inverses (lines of
                // f.ikmask: i k_x times the input, the x derivative); out: u x omega, tau
  double invN;
  double csd2;
  const MlpPacked* mlp;
};

// nu_t -> u x omega (from omega = (A_zy - A_yz, A_xz - A_zx, A_yx - A_xy)) and
// tau = 2 nu_t S (xx, yy, zz, xy, xz, yz) of one point; A_ij at index 3 i + j.
template <typename T>
__device__ __forceinline__ void closure_point(const cx_t<T> (&u)[3], const cx_t<T> (&A)[9], T nu,
                                              cx_t<T> (&o)[9]) {
  const cx_t<T> w0 = csub(A[7], A[5]), w1 = csub(A[2], A[6]), w2 = csub(A[3], A[1]);
  o[0] = csub(cmul(u[1], w2), cmul(u[2], w1));
  o[1] = csub(cmul(u[2], w0), cmul(u[0], w2));
  o[2] = csub(cmul(u[0], w1), cmul(u[1], w0));
  o[3] = cscale((T)2 * nu, A[0]);
  o[4] = cscale((T)2 * nu, A[4]);
  o[5] = cscale((T)2 * nu, A[8]);
  o[6] = cscale(nu, cadd(A[1], A[3]));
  o[7] = cscale(nu, cadd(A[2], A[6]));
  o[8] = cscale(nu, cadd(A[5], A[7]));
}

// The closure's x pass: x-inverse of the 12 fields of G rows into shared
// memory, nu_t per point (the MLP as four 128-point tcgen05 tiles, or
// Smagorinsky (Cs Delta)^2 sqrt(2 S:S) from the real gradient), u x omega and
// tau written over the rows, x-forward of the 9 results.  Rows are
// field-major (line = field * G + row), so the warps that hold only the
// three discarded gradient fields skip the forward transform.
template <typename T, int L, int MODEL>
__global__ void __launch_bounds__(kXlesThreads)
    k_xles(const XlesArgs a, const cx_t<T>* __restrict__ tw) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL, RS = xrow_stride(L, (int)sizeof(C));
  constexpr int G = 32 / TPL;
  constexpr int PTS = G * L;
  static_assert(TPL <= 32 && 12 * G * TPL == kXlesThreads, "tile shape");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  using MS = typename std::conditional<MODEL == CLOSURE_MLP, XlesTcSmem, XlesNoSmem>::type;
  __shared__ MS S;
  __shared__ float nus[PTS];
  const int64_t row0 = (int64_t)blockIdx.x * G;
  const int j = threadIdx.x % TPL, line = threadIdx.x / TPL;
  const int fld = line / G, gl = line - fld * G;
  C* row = sm + line * RS;
  pdl_trigger();
  // the model does not depend on the previous launch: load it before the wait
  if constexpr (MODEL == CLOSURE_MLP) {
    mlp_tc_load_weights(a.mlp, S.W1, S.W2, S.B2, S.w3, threadIdx.x, blockDim.x);
    mlp_tc_fill_ones(S.ONES, 128, threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) {
      S.b3 = a.mlp->b3;
      S.s_in = a.mlp->s_in;
      S.s_out = a.mlp->s_out;
      S.abort = 0;
      tc::mbar_init(&S.mbar, 1);
    }
    if (threadIdx.x < 32) {
      tc::tmem_alloc(&S.tmem, 64);
      tc::tmem_relinquish();
    }
  }
  pdl_wait();
  C v[E];
  {
    const C* __restrict__ src = reinterpret_cast<const C*>(select_ptr(a.f.in, fld));
    const int64_t i0 = (row0 + gl) * L + j;
    const bool ik = (a.f.ikmask >> fld) & 1u;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const C x = src[i0 + TPL * e];
      v[e] = ik ? ikmul((T)freq_i(j + TPL * e, L), x) : x;
    }
  }
  line_fft<L>(v, row, j, tw, (T)1);
#pragma unroll
  for (int e = 0; e < E; e++) row[pad_pos(j + TPL * e)] = v[e];
  if constexpr (MODEL == CLOSURE_MLP) tc::fence_before_sync();
  __syncthreads();
  if constexpr (MODEL == CLOSURE_MLP) tc::fence_after_sync();

  const T invN = (T)a.invN;
  auto at = [&](int field, int p) -> C& {
    return sm[(field * G + p / L) * RS + pad_pos(p % L)];
  };
  if constexpr (MODEL == CLOSURE_MLP) {
    const int tid = threadIdx.x, warp = tid >> 5;
    if (warp < 4) {
      const uint32_t tmem = S.tmem;
      const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
      const uint32_t sX = tc::smem_u32(S.X), sH = tc::smem_u32(S.H), sO = tc::smem_u32(S.ONES);
      const uint32_t sW1 = tc::smem_u32(S.W1), sW2 = tc::smem_u32(S.W2),
                     sB2 = tc::smem_u32(S.B2);
      constexpr uint32_t id = tc::idesc_bf16(128, kMlpHidden);
      const float s_in = S.s_in;
      const uint32_t one2 = bf16_bits(1.f) * 0x10001u;
      uint32_t phase = 0;
      for (int tile = 0; tile < PTS / 128; tile++) {
        const int p = 128 * tile + tid;
        // features s_in Re(A_ij) / N (columns 0..8), the bias columns 9, 10 = 1
        {
          float fv[kMlpIn];
#pragma unroll
          for (int q = 0; q < kMlpIn; q++) fv[q] = (float)(at(3 + q, p).x * invN) * s_in;
          const uint4 x0 = make_uint4(pack_bf16(fv[0], fv[1]), pack_bf16(fv[2], fv[3]),
                                      pack_bf16(fv[4], fv[5]), pack_bf16(fv[6], fv[7]));
          const uint4 x1 = make_uint4((bf16_bits(fv[8]) & 0xFFFFu) | (one2 & 0xFFFF0000u),
                                      one2 & 0xFFFFu, 0u, 0u);
          *reinterpret_cast<uint4*>(S.X + tc::kmajor_off(tid, 0, kMlpK1)) = x0;
          *reinterpret_cast<uint4*>(S.X + tc::kmajor_off(tid, 8, kMlpK1)) = x1;
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        mlp_warps_sync();
        if (tid == 0) {
          tc::fence_after_sync();
          tc::mma_bf16(tmem, tc::sdesc(sX, 128, 16 * kMlpK1), tc::sdesc(sW1, 128, 16 * kMlpK1),
                       id, 0);
          tc::commit(&S.mbar);
        }
        if (!tc::mbar_wait(&S.mbar, phase, tc::kWaitCycles)) S.abort = 1;
        phase ^= 1;
        tc::fence_after_sync();
        mlp_warps_sync();
        if (S.abort) break;
#pragma unroll
        for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
          uint32_t r[16];
          tc::tmem_ld16(tmem + lane_base + c0, r);
          uint32_t h[8];
#pragma unroll
          for (int q = 0; q < 8; q++)
            h[q] = pack_bf16(fmaxf(__uint_as_float(r[2 * q]), 0.f),
                             fmaxf(__uint_as_float(r[2 * q + 1]), 0.f));
          *reinterpret_cast<uint4*>(S.H + tc::kmajor_off(tid, c0, kMlpHidden)) =
              make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4*>(S.H + tc::kmajor_off(tid, c0 + 8, kMlpHidden)) =
              make_uint4(h[4], h[5], h[6], h[7]);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        mlp_warps_sync();
        if (tid == 0) {
          tc::fence_after_sync();
#pragma unroll
          for (int s = 0; s < kMlpHidden / 16; s++)
            tc::mma_bf16(tmem, tc::sdesc(sH + 256 * s, 128, 16 * kMlpHidden),
                         tc::sdesc(sW2 + 256 * s, 128, 16 * kMlpHidden), id, s > 0);
          tc::mma_bf16(tmem, tc::sdesc(sO, 128, 256), tc::sdesc(sB2, 128, 256), id, 1);
          tc::commit(&S.mbar);
        }
        if (!tc::mbar_wait(&S.mbar, phase, tc::kWaitCycles)) S.abort = 1;
        phase ^= 1;
        tc::fence_after_sync();
        mlp_warps_sync();
        if (S.abort) break;
        float z = 0.f;
#pragma unroll
        for (int c0 = 0; c0 < kMlpHidden; c0 += 16) {
          uint32_t r[16];
          tc::tmem_ld16(tmem + lane_base + c0, r);
#pragma unroll
          for (int q = 0; q < 16; q++) z += fmaxf(__uint_as_float(r[q]), 0.f) * S.w3[c0 + q];
        }
        nus[p] = S.s_out * softplus_f(z + S.b3);
        tc::fence_before_sync();
      }
      if (S.abort) {
        // an MMA whose wait ran out may still be in flight: one more bounded wait
        tc::mbar_wait(&S.mbar, phase ^ 1, tc::kWaitCycles);
        if (tid == 0) atomicExch(&g_xles_tc_status, 1);
      }
      tc::fence_before_sync();
      mlp_warps_sync();
      if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 64);
      }
    }
    __syncthreads();
  }
  for (int p = threadIdx.x; p < PTS; p += kXlesThreads) {
    C u[3], A[9], o[9];
#pragma unroll
    for (int d = 0; d < 3; d++) u[d] = cscale(invN, at(d, p));
#pragma unroll
    for (int q = 0; q < 9; q++) A[q] = cscale(invN, at(3 + q, p));
    T nu;
    if constexpr (MODEL == CLOSURE_MLP) {
      nu = (T)nus[p];
    } else {
      T s2 = 0;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int jj = 0; jj < 3; jj++) {
          const T sij = (T)0.5 * (A[3 * i + jj].x + A[3 * jj + i].x);
          s2 += sij * sij;
        }
      nu = (T)a.csd2 * sqrt((T)2 * s2);
    }
    closure_point<T>(u, A, nu, o);
#pragma unroll
    for (int q = 0; q < 9; q++) at(q, p) = o[q];
  }
  __syncthreads();

  constexpr int kLinesPerWarp = 32 / TPL;
  const bool skip = ((9 * G) % kLinesPerWarp == 0) && fld >= 9;
  if (!skip) {
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = row[pad_pos(j + TPL * e)];
    line_sync<TPL>();
    line_fft<L>(v, row, j, tw, (T)-1);
  }
  if (fld < 9) {
    C* __restrict__ dst = reinterpret_cast<C*>(select_ptr(a.f.out, fld));
    const int64_t i0 = (row0 + gl) * L + j;
#pragma unroll
    for (int e = 0; e < E; e++) dst[i0 + TPL * e] = v[e];
  }
}

template <typename T, int L, int MODEL>
int launch_xles_l(const XlesArgs& a, int64_t rows, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr int TPL = LinePlan<L>::TPL;
  constexpr int G = 32 / TPL;
  if (rows % G) {
    set_error("closure step: ny * nz must be a multiple of the x-pass rows per CTA");
    return ERR_UNSUPPORTED;
  }
  const size_t smem = (size_t)12 * G * xrow_stride(L, (int)sizeof(C)) * sizeof(C);
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = allow_max_dynamic_smem(k_xles<T, L, MODEL>);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_xles)");
    attr[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  cudaError_t e = launch_pdl(k_xles<T, L, MODEL>, dim3((unsigned)(rows / G)), dim3(kXlesThreads),
                             smem, s, a, tw);
  if (e != cudaSuccess) return cuda_status(e, "k_xles");
  return OK;
}

template <typename T, int MODEL>
int launch_xles_m(const XlesArgs& a, int nx, int64_t rows, cudaStream_t s) {
  switch (nx) {
    case 16: return launch_xles_l<T, 16, MODEL>(a, rows, s);
    case 32: return launch_xles_l<T, 32, MODEL>(a, rows, s);
    case 64: return launch_xles_l<T, 64, MODEL>(a, rows, s);
    case 128: return launch_xles_l<T, 128, MODEL>(a, rows, s);
    case 256: return launch_xles_l<T, 256, MODEL>(a, rows, s);
    default:
      set_error("closure step: nx must be a power of two in [16, 256]");
      return ERR_UNSUPPORTED;
  }
}

template <typename T>
int launch_xles(const XlesArgs& a, int model, int nx, int64_t rows, cudaStream_t s) {
  return model == CLOSURE_MLP ? launch_xles_m<T, CLOSURE_MLP>(a, nx, rows, s)
                              : launch_xles_m<T, CLOSURE_SMAGORINSKY>(a, nx, rows, s);
}

int les_tc_status_take(int* timed_out) {
  int v = 0;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpyFromSymbol(&v, g_xles_tc_status, sizeof(int));
  if (e == cudaSuccess && v) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_xles_tc_status, &zero, sizeof(int));
  }
  *timed_out = v;
  return cuda_status(e, "les_tc_status_take");
}

int les_step_once(const NSPlan& pl, void* const V[3], void* const C0[3], void* const U[kLESWork],
                  double* stats, double nu, double dt, const Closure& cl, cudaStream_t s) {
  const int nx = pl.nx, ny = pl.ny, nz = pl.nz, prec = pl.prec;
  const int64_t n = (int64_t)nx * ny * nz;
  if (n % 32) {
    set_error("closure step: nx*ny*nz must be a multiple of 32");
    return ERR_UNSUPPORTED;
  }
  if (cl.model == CLOSURE_MLP && !cl.mlp) {
    set_error("closure step: no MLP model set");
    return ERR_ARG;
  }
  const PdlScope pdl;  // the five launches overlap their neighbours' edges
  int rc;
  auto pass = [&](int axis, const FieldPtrs& f, int sign, int pro) -> int {
    LineGeo g = axis_geo(axis, nx, ny, nz, prec, pl.lineW);
    return run_line_pass(g, f, sign, 0, 1.0, prec, s, pro);
  };
  // z-inverse: U[0..2] = V, U[3..5] = d_z V
  {
    FieldPtrs f{};
    f.n = 6;
    for (int q = 0; q < 6; q++) {
      f.in[q] = V[q % 3];
      f.out[q] = U[q];
    }
    f.ikmask = 0x38u;
    if ((rc = pass(2, f, +1, PRO_IKAXIS))) return rc;
  }
  // y-inverse: U[6..8] = V, U[3..5] = d_z V (in place), U[9..11] = d_y V;
  // U[0..2] is only read
  {
    FieldPtrs f{};
    f.n = 9;
    for (int i = 0; i < 3; i++) {
      f.in[i] = U[i];
      f.out[i] = U[6 + i];
      f.in[3 + i] = U[3 + i];
      f.out[3 + i] = U[3 + i];
      f.in[6 + i] = U[i];
      f.out[6 + i] = U[9 + i];
    }
    f.ikmask = 0x1C0u;
    if ((rc = pass(1, f, +1, PRO_IKAXIS))) return rc;
  }
  // x-inverse (line 3 + 3 i + 0 = d_x V_i from U[6 + i]), closure, x-forward
  // of u x omega (into U[0..2]) and tau (U[3..8]); every CTA reads its rows
  // of all inputs before it writes them
  {
    XlesArgs a{};
    a.f.n = kLESWork;
    for (int i = 0; i < 3; i++) {
      a.f.in[i] = U[6 + i];
      a.f.in[3 + 3 * i + 0] = U[6 + i];
      a.f.in[3 + 3 * i + 1] = U[9 + i];
      a.f.in[3 + 3 * i + 2] = U[3 + i];
      a.f.ikmask |= 1u << (3 + 3 * i);
    }
    for (int q = 0; q < kLESWork; q++) a.f.out[q] = U[q];
    a.invN = 1.0 / (double)n;
    a.csd2 = cl.csd2;
    a.mlp = reinterpret_cast<const MlpPacked*>(cl.mlp);
    const int64_t rows = (int64_t)ny * nz;
    rc = prec == PREC_C128 ? launch_xles<double>(a, cl.model, nx, rows, s)
                           : launch_xles<float>(a, cl.model, nx, rows, s);
    if (rc) return rc;
  }
  // y-forward of the 9 results
  {
    FieldPtrs f{};
    f.n = 9;
    for (int q = 0; q < 9; q++) f.in[q] = f.out[q] = U[q];
    if ((rc = pass(1, f, -1, PRO_LOAD))) return rc;
  }
  // z-forward of u x omega + div tau + update
  UpdateArgs a{};
  for (int d = 0; d < 3; d++) {
    a.U[d] = U[d];
    a.V[d] = V[d];
    a.C0[d] = C0[d];
  }
  for (int q = 0; q < 6; q++) a.tau[q] = U[3 + q];
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.lx = 0;
  while ((1 << a.lx) < nx) a.lx++;
  a.W = pl.sgs_W;
  a.hK = dt / 2;
  a.nuhK = nu * dt / 2;
  a.stats = stats;
  a.kc2 = pl.kc2;
  a.sgs_klo = pl.sgs_klo;
  a.sgs_kinv = pl.sgs_kinv;
  return ns_update(pl, a, true, s);
}

// ---------------------------------------------------------------------------
// data kernels

// Sharp spherical cutoff |k| <= kc of fine fields (nf^3) onto nc^3 grids,
// scaled by nc^3 / nf^3 (the unnormalised DFT of the coarse grid).
template <typename T>
__global__ void k_truncate(FieldPtrs f, int nf, int nc, double kc2, T scale) {
  using C = cx_t<T>;
  const int fld = blockIdx.y;
  const C* __restrict__ in = reinterpret_cast<const C*>(f.in[fld]);
  C* __restrict__ out = reinterpret_cast<C*>(f.out[fld]);
  const int64_t n3 = (int64_t)nc * nc * nc;
  const int h = nc >> 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i % nc), iy = (int)((i / nc) % nc), iz = (int)(i / ((int64_t)nc * nc));
    const int kx = freq_i(ix, nc), ky = freq_i(iy, nc), kz = freq_i(iz, nc);
    const bool keep = (double)kx * kx + (double)ky * ky + (double)kz * kz <= kc2 &&
                      abs(kx) < h && abs(ky) < h && abs(kz) < h;
    C v = mk((T)0, (T)0);
    if (keep) {
      const int64_t fx = kx < 0 ? kx + nf : kx, fy = ky < 0 ? ky + nf : ky,
                    fz = kz < 0 ? kz + nf : kz;
      v = cscale(scale, in[fx + (int64_t)nf * (fy + (int64_t)nf * fz)]);
    }
    out[i] = v;
  }
}

// Coarse fields (nc^3) onto fine grids (nf^3), zero outside, scaled by
// nf^3 / nc^3.
template <typename T>
__global__ void k_pad(FieldPtrs f, int nc, int nf, T scale) {
  using C = cx_t<T>;
  const int fld = blockIdx.y;
  const C* __restrict__ in = reinterpret_cast<const C*>(f.in[fld]);
  C* __restrict__ out = reinterpret_cast<C*>(f.out[fld]);
  const int64_t n3 = (int64_t)nf * nf * nf;
  const int h = nc >> 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i % nf), iy = (int)((i / nf) % nf), iz = (int)(i / ((int64_t)nf * nf));
    const int kx = freq_i(ix, nf), ky = freq_i(iy, nf), kz = freq_i(iz, nf);
    C v = mk((T)0, (T)0);
    if (abs(kx) < h && abs(ky) < h && abs(kz) < h) {
      const int64_t cx = kx < 0 ? kx + nc : kx, cy = ky < 0 ? ky + nc : ky,
                    cz = kz < 0 ? kz + nc : kz;
      v = cscale(scale, in[cx + (int64_t)nc * (cy + (int64_t)nc * cz)]);
    }
    out[i] = v;
  }
}

// T_q = u_i u_j - ub_i ub_j for q = xx, yy, zz, xy, xz, yz (physical fields).
template <typename T>
__global__ void k_sgs_products(FieldPtrs uu, FieldPtrs tt, int64_t n) {
  using C = cx_t<T>;
  const int I[6] = {0, 1, 2, 0, 0, 1}, J[6] = {0, 1, 2, 1, 2, 2};
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    C u[3], ub[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      u[d] = reinterpret_cast<const C*>(uu.in[d])[p];
      ub[d] = reinterpret_cast<const C*>(uu.in[3 + d])[p];
    }
#pragma unroll
    for (int q = 0; q < 6; q++)
      reinterpret_cast<C*>(tt.out[q])[p] = csub(cmul(u[I[q]], u[J[q]]), cmul(ub[I[q]], ub[J[q]]));
  }
}

struct TargetArgs {
  const void* A[9];    // filtered velocity gradient (physical, coarse)
  const void* tau[6];  // filtered SGS stress (physical, coarse)
  int64_t n;
  double s_in;
  __nv_bfloat16* X;  // [n][16]
  float* nut;        // [n]
  float* weight;     // [n] S:S (may be null)
};

// Features s_in * Re A (padded to 16) and the pointwise least-squares eddy
// viscosity nu_t = -(tau^d : S) / (2 S : S) of the filtered SGS stress.
template <typename T>
__global__ void k_sgs_target(const TargetArgs a) {
  using C = cx_t<T>;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.n;
       p += (int64_t)gridDim.x * blockDim.x) {
    double A[9], t6[6];
#pragma unroll
    for (int q = 0; q < 9; q++) A[q] = (double)reinterpret_cast<const C*>(a.A[q])[p].x;
#pragma unroll
    for (int q = 0; q < 6; q++) t6[q] = (double)reinterpret_cast<const C*>(a.tau[q])[p].x;
    const double tr = (t6[0] + t6[1] + t6[2]) / 3.0;
    const double Sxx = A[0], Syy = A[4], Szz = A[8];
    const double Sxy = 0.5 * (A[1] + A[3]), Sxz = 0.5 * (A[2] + A[6]), Syz = 0.5 * (A[5] + A[7]);
    const double num = (t6[0] - tr) * Sxx + (t6[1] - tr) * Syy + (t6[2] - tr) * Szz +
                       2.0 * (t6[3] * Sxy + t6[4] * Sxz + t6[5] * Syz);
    const double den = Sxx * Sxx + Syy * Syy + Szz * Szz + 2.0 * (Sxy * Sxy + Sxz * Sxz + Syz * Syz);
    a.nut[p] = (float)(-num / (2.0 * den + 1e-30));
    if (a.weight) a.weight[p] = (float)den;
    __nv_bfloat16* row = a.X + p * kMlpK1;
#pragma unroll
    for (int q = 0; q < kMlpK1; q++)
      row[q] = __float2bfloat16_rn(q < kMlpIn ? (float)(A[q] * a.s_in) : 0.f);
  }
}

// Shell sums E(round |k|) += |V|^2 * scale, shells < nshell.
template <typename T>
__global__ void k_spectrum(FieldPtrs f, int nx, int ny, int nz, double scale, double* E,
                           int nshell) {
  using C = cx_t<T>;
  extern __shared__ double hist[];
  for (int i = threadIdx.x; i < nshell; i += blockDim.x) hist[i] = 0.0;
  __syncthreads();
  const int64_t n = (int64_t)nx * ny * nz;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((int64_t)nx * ny));
    const double kx = freq_i(ix, nx), ky = freq_i(iy, ny), kz = freq_i(iz, nz);
    const int sh = (int)rint(sqrt(kx * kx + ky * ky + kz * kz));
    double e = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const C v = reinterpret_cast<const C*>(f.in[d])[i];
      e += (double)v.x * v.x + (double)v.y * v.y;
    }
    if (sh < nshell) atomicAdd(&hist[sh], e * scale);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nshell; i += blockDim.x)
    if (hist[i] != 0.0) atomicAdd(&E[i], hist[i]);
}

namespace {

inline int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

bool fields_ok(const void* const* p, int n, const char* what) {
  if (!p) {
    set_error(std::string(what) + ": null field array");
    return false;
  }
  for (int i = 0; i < n; i++)
    if (!p[i]) {
      set_error(std::string(what) + ": null field pointer");
      return false;
    }
  return true;
}

int truncate_fields(const void* const* in, void* const* out, int nf_fields, int nf, int nc,
                    double kc, int prec, cudaStream_t s) {
  FieldPtrs f{};
  f.n = nf_fields;
  for (int i = 0; i < nf_fields; i++) {
    f.in[i] = const_cast<void*>(in[i]);
    f.out[i] = out[i];
  }
  const dim3 grid(grid_for((int64_t)nc * nc * nc), nf_fields);
  const double scale = (double)nc * nc * nc / ((double)nf * nf * nf);
  if (prec == PREC_C128)
    k_truncate<double><<<grid, 256, 0, s>>>(f, nf, nc, kc * kc, scale);
  else
    k_truncate<float><<<grid, 256, 0, s>>>(f, nf, nc, kc * kc, (float)scale);
  SNS_CHECK_LAUNCH("k_truncate");
  return OK;
}

int pad_fields(const void* const* in, void* const* out, int nfields, int nc, int nf, int prec,
               cudaStream_t s) {
  FieldPtrs f{};
  f.n = nfields;
  for (int i = 0; i < nfields; i++) {
    f.in[i] = const_cast<void*>(in[i]);
    f.out[i] = out[i];
  }
  const dim3 grid(grid_for((int64_t)nf * nf * nf), nfields);
  const double scale = (double)nf * nf * nf / ((double)nc * nc * nc);
  if (prec == PREC_C128)
    k_pad<double><<<grid, 256, 0, s>>>(f, nc, nf, scale);
  else
    k_pad<float><<<grid, 256, 0, s>>>(f, nc, nf, (float)scale);
  SNS_CHECK_LAUNCH("k_pad");
  return OK;
}

bool cube_ok(int64_t nf, int64_t nc, const char* what) {
  if (!is_pow2(nf) || !is_pow2(nc) || nc > nf || nc < 4 || nf > 1024) {
    set_error(std::string(what) + ": grids must be powers of two with 4 <= nc <= nf <= 1024");
    return false;
  }
  return true;
}

}  // namespace
}  // namespace sns

using namespace sns;

extern "C" {

int sns_spectral_truncate(const void* const* in, void* const* out, int nfields, int64_t nf,
                          int64_t nc, double kc, int prec, void* stream) {
  if (nfields < 1 || nfields > kMaxFields || !fields_ok(in, nfields, "sns_spectral_truncate") ||
      !fields_ok((const void* const*)out, nfields, "sns_spectral_truncate") ||
      (prec != PREC_C64 && prec != PREC_C128)) {
    if (nfields < 1 || nfields > kMaxFields) set_error("sns_spectral_truncate: 1..12 fields");
    if (prec != PREC_C64 && prec != PREC_C128) set_error("sns_spectral_truncate: bad precision");
    return ERR_ARG;
  }
  if (!cube_ok(nf, nc, "sns_spectral_truncate")) return ERR_UNSUPPORTED;
  return truncate_fields(in, out, nfields, (int)nf, (int)nc, kc, prec,
                         reinterpret_cast<cudaStream_t>(stream));
}

int sns_spectral_pad(const void* const* in, void* const* out, int nfields, int64_t nc, int64_t nf,
                     int prec, void* stream) {
  if (nfields < 1 || nfields > kMaxFields || !fields_ok(in, nfields, "sns_spectral_pad") ||
      !fields_ok((const void* const*)out, nfields, "sns_spectral_pad") ||
      (prec != PREC_C64 && prec != PREC_C128)) {
    if (nfields < 1 || nfields > kMaxFields) set_error("sns_spectral_pad: 1..12 fields");
    if (prec != PREC_C64 && prec != PREC_C128) set_error("sns_spectral_pad: bad precision");
    return ERR_ARG;
  }
  if (!cube_ok(nf, nc, "sns_spectral_pad")) return ERR_UNSUPPORTED;
  return pad_fields(in, out, nfields, (int)nc, (int)nf, prec,
                    reinterpret_cast<cudaStream_t>(stream));
}

int sns_sgs_sample(const void* const V[3], int64_t nf, int64_t nc, double kc, double s_in,
                   int prec, void* X, float* nut, float* weight, void* const Vc_out[3],
                   void* stream) {
  if (!fields_ok(V, 3, "sns_sgs_sample") || !X || !nut ||
      (prec != PREC_C64 && prec != PREC_C128)) {
    if (!X || !nut) set_error("sns_sgs_sample: null output");
    if (prec != PREC_C64 && prec != PREC_C128) set_error("sns_sgs_sample: bad precision");
    return ERR_ARG;
  }
  if (!cube_ok(nf, nc, "sns_sgs_sample")) return ERR_UNSUPPORTED;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t esz = prec == PREC_C128 ? 16 : 8;
  const int64_t nf3 = nf * nf * nf, nc3 = nc * nc * nc;
  // work: 12 fine fields (u, ubar, T) and 18 coarse fields (Vc, tau, A)
  void* fine[12] = {};
  void* coarse[18] = {};
  int rc = OK;
  for (int i = 0; i < 12 && !rc; i++) rc = pool_malloc(&fine[i], esz * nf3);
  for (int i = 0; i < 18 && !rc; i++) rc = pool_malloc(&coarse[i], esz * nc3);
  auto release = [&]() {
    cudaStreamSynchronize(s);
    for (void* p : fine) pool_free(p);
    for (void* p : coarse) pool_free(p);
  };
  if (rc) {
    release();
    return rc;
  }
  void** Vc = &coarse[0];
  void** tau = &coarse[3];
  void** A = &coarse[9];
  void** u = &fine[0];
  void** ub = &fine[3];
  void** T = &fine[6];
  const int Nf = (int)nf, Nc = (int)nc;
  do {
    if ((rc = truncate_fields(V, Vc, 3, Nf, Nc, kc, prec, s))) break;
    if ((rc = pad_fields((const void* const*)Vc, ub, 3, Nc, Nf, prec, s))) break;
    if ((rc = fft3d(ub, 3, Nf, Nf, Nf, +1, PASS_SCALE, prec, s))) break;
    for (int d = 0; d < 3 && !rc; d++)
      rc = cuda_status(cudaMemcpyAsync(u[d], V[d], esz * nf3, cudaMemcpyDeviceToDevice, s),
                       "sns_sgs_sample");
    if (rc) break;
    if ((rc = fft3d(u, 3, Nf, Nf, Nf, +1, PASS_SCALE, prec, s))) break;
    {
      FieldPtrs uu{}, tt{};
      for (int d = 0; d < 3; d++) {
        uu.in[d] = u[d];
        uu.in[3 + d] = ub[d];
      }
      for (int q = 0; q < 6; q++) tt.out[q] = T[q];
      if (prec == PREC_C128)
        k_sgs_products<double><<<grid_for(nf3), 256, 0, s>>>(uu, tt, nf3);
      else
        k_sgs_products<float><<<grid_for(nf3), 256, 0, s>>>(uu, tt, nf3);
      if ((rc = cuda_status(cudaGetLastError(), "k_sgs_products"))) break;
    }
    if ((rc = fft3d(T, 6, Nf, Nf, Nf, -1, 0, prec, s))) break;
    if ((rc = truncate_fields((const void* const*)T, tau, 6, Nf, Nc, kc, prec, s))) break;
    if ((rc = fft3d(tau, 6, Nc, Nc, Nc, +1, PASS_SCALE, prec, s))) break;
    const Dims dc{Nc, Nc, Nc};
    for (int i = 0; i < 3 && !rc; i++)
      rc = op_gradient(Vc[i], A[3 * i], A[3 * i + 1], A[3 * i + 2], dc, prec, s);
    if (rc) break;
    if ((rc = fft3d(A, 6, Nc, Nc, Nc, +1, PASS_SCALE, prec, s))) break;
    if ((rc = fft3d(A + 6, 3, Nc, Nc, Nc, +1, PASS_SCALE, prec, s))) break;
    TargetArgs ta{};
    for (int q = 0; q < 9; q++) ta.A[q] = A[q];
    for (int q = 0; q < 6; q++) ta.tau[q] = tau[q];
    ta.n = nc3;
    ta.s_in = s_in;
    ta.X = reinterpret_cast<__nv_bfloat16*>(X);
    ta.nut = nut;
    ta.weight = weight;
    if (prec == PREC_C128)
      k_sgs_target<double><<<grid_for(nc3), 256, 0, s>>>(ta);
    else
      k_sgs_target<float><<<grid_for(nc3), 256, 0, s>>>(ta);
    if ((rc = cuda_status(cudaGetLastError(), "k_sgs_target"))) break;
    if (Vc_out)
      for (int d = 0; d < 3 && !rc; d++)
        if (Vc_out[d])
          rc = cuda_status(
              cudaMemcpyAsync(Vc_out[d], Vc[d], esz * nc3, cudaMemcpyDeviceToDevice, s),
              "sns_sgs_sample");
  } while (false);
  release();
  return rc;
}

int sns_energy_spectrum(const void* const V[3], int64_t nx, int64_t ny, int64_t nz, int prec,
                        double* E, int nshell, void* stream) {
  if (!fields_ok(V, 3, "sns_energy_spectrum") || !E || nshell < 1 || nshell > 4096 ||
      (prec != PREC_C64 && prec != PREC_C128)) {
    if (!E || nshell < 1 || nshell > 4096) set_error("sns_energy_spectrum: bad output");
    if (prec != PREC_C64 && prec != PREC_C128) set_error("sns_energy_spectrum: bad precision");
    return ERR_ARG;
  }
  if (nx < 1 || ny < 1 || nz < 1 || nx * ny * nz >= ((int64_t)1 << 32)) {
    set_error("sns_energy_spectrum: dimensions out of range");
    return ERR_ARG;
  }
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int rc = cuda_status(cudaMemsetAsync(E, 0, sizeof(double) * nshell, s), "sns_energy_spectrum");
  if (rc) return rc;
  FieldPtrs f{};
  for (int d = 0; d < 3; d++) f.in[d] = const_cast<void*>(V[d]);
  const double N = (double)nx * ny * nz;
  const double scale = 1.0 / (2.0 * N * N);
  const int grid = grid_for(nx * ny * nz);
  const size_t smem = sizeof(double) * nshell;
  if (prec == PREC_C128)
    k_spectrum<double><<<grid, 256, smem, s>>>(f, (int)nx, (int)ny, (int)nz, scale, E, nshell);
  else
    k_spectrum<float><<<grid, 256, smem, s>>>(f, (int)nx, (int)ny, (int)nz, scale, E, nshell);
  SNS_CHECK_LAUNCH("k_spectrum");
  return OK;
}

}  // extern "C"
