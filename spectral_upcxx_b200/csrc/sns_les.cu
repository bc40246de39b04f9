// Eddy-viscosity closure of the fused NS step, and the data kernels of the
// learned closure (spectral filter, SGS targets, energy spectrum).
//
// No reference counterpart: exec/ns.cpp has no subgrid model.  The closure
// step adds the divergence of the eddy stress tau_ij = 2 nu_t S_ij to the
// nonlinear term cross1 (ns.cpp:203-206) and is otherwise the ns.cpp step:
//
//   z-inverse of V and grad V (i k_j V_i)   1 launch x 12 fields
//   y-inverse                               1 x 12
//   x-inverse                               1 x 12
//   closure: nu_t (Smagorinsky or the MLP on the tensor cores), u x omega
//            and tau_ij pointwise           1
//   x-forward, y-forward of u x omega, tau  2 x 9
//   z-forward of tau                        1 x 6
//   z-forward of u x omega + i k_j tau_ij + the AB2 / projection / CN
//   update                                  1
#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>
#include <string>

#include "../../include/spectral_b200.h"
#include "sns_ens.cuh"
#include "sns_fft.cuh"
#include "sns_les.cuh"
#include "sns_mlp.cuh"
#include "sns_ops.cuh"
#include "sns_tiles.cuh"

namespace sns {

constexpr int kClWarps = 8;
constexpr int kXsStride = 24;  // bf16 per feature row (bank-spread A loads)

struct ClosureArgs {
  void* U[kLESWork];  // in: u (3), A_ij = d_j u_i (9), unnormalised; out: u x omega, tau
  int64_t n;
  double invN;
  double csd2;
  const MlpPacked* mlp;
};

// Per point: nu_t, omega and u x omega from the velocity gradient, tau_ij =
// 2 nu_t S_ij.  Warps take 32 points; with the MLP, a warp evaluates its
// points as two 16-row tiles on the tensor cores.
template <typename T, int MODEL>
__global__ void __launch_bounds__(kClWarps * 32) k_les_closure(const ClosureArgs a) {
  using C = cx_t<T>;
  __shared__ MlpSmem S;
  __shared__ __align__(16) __nv_bfloat16 xs[kClWarps][32 * kXsStride];
  __shared__ float nus[kClWarps][32];
  if constexpr (MODEL == CLOSURE_MLP) {
    mlp_load_smem(a.mlp, S, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const T invN = (T)a.invN;
  const C* __restrict__ in[kLESWork];
#pragma unroll
  for (int q = 0; q < kLESWork; q++) in[q] = reinterpret_cast<const C*>(a.U[q]);
  for (int64_t p0 = ((int64_t)blockIdx.x * kClWarps + warp) * 32; p0 < a.n;
       p0 += (int64_t)gridDim.x * kClWarps * 32) {
    const int64_t p = p0 + lane;
    T nu = 0;
    if constexpr (MODEL == CLOSURE_MLP) {
      __nv_bfloat16* row = &xs[warp][lane * kXsStride];
#pragma unroll
      for (int q = 0; q < kMlpIn; q++)
        row[q] = __float2bfloat16_rn((float)(in[3 + q][p].x * invN) * S.s_in);
#pragma unroll
      for (int q = kMlpIn; q < kMlpK1; q++) row[q] = __float2bfloat16_rn(0.f);
      __syncwarp();
#pragma unroll
      for (int m = 0; m < 2; m++) {
        uint32_t xa[4];
        load_a_tile(&xs[warp][16 * m * kXsStride], kXsStride, xa);
        MlpTile tile;
        mlp_tile_forward<false>(S, xa, tile);
        if ((lane & 3) == 0) {
          const int g = lane >> 2;
          nus[warp][16 * m + g] = S.s_out * softplus_f(tile.z[0]);
          nus[warp][16 * m + g + 8] = S.s_out * softplus_f(tile.z[1]);
        }
      }
      __syncwarp();
      nu = (T)nus[warp][lane];
    }
    C A[9], u[3];
#pragma unroll
    for (int q = 0; q < 9; q++) A[q] = cscale(invN, in[3 + q][p]);
#pragma unroll
    for (int d = 0; d < 3; d++) u[d] = cscale(invN, in[d][p]);
    if constexpr (MODEL == CLOSURE_SMAGORINSKY) {
      // (Cs Delta)^2 sqrt(2 S:S), S from the real gradient
      T s2 = 0;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
          const T sij = (T)0.5 * (A[3 * i + j].x + A[3 * j + i].x);
          s2 += sij * sij;
        }
      nu = (T)a.csd2 * sqrt((T)2 * s2);
    }
    // omega = (A_zy - A_yz, A_xz - A_zx, A_yx - A_xy), A_ij at 3 i + j
    const C w0 = csub(A[7], A[5]), w1 = csub(A[2], A[6]), w2 = csub(A[3], A[1]);
    C* __restrict__ out[9];
#pragma unroll
    for (int q = 0; q < 9; q++) out[q] = reinterpret_cast<C*>(a.U[q]);
    out[0][p] = csub(cmul(u[1], w2), cmul(u[2], w1));
    out[1][p] = csub(cmul(u[2], w0), cmul(u[0], w2));
    out[2][p] = csub(cmul(u[0], w1), cmul(u[1], w0));
    // tau = 2 nu S: xx, yy, zz, xy, xz, yz
    out[3][p] = cscale((T)2 * nu, A[0]);
    out[4][p] = cscale((T)2 * nu, A[4]);
    out[5][p] = cscale((T)2 * nu, A[8]);
    out[6][p] = cscale(nu, cadd(A[1], A[3]));
    out[7][p] = cscale(nu, cadd(A[2], A[6]));
    out[8][p] = cscale(nu, cadd(A[5], A[7]));
  }
}

template <typename T>
int launch_closure(const ClosureArgs& a, int model, cudaStream_t s) {
  // MLP: a resident grid (two CTAs per SM), so each CTA loads the weights once
  const int64_t groups = a.n / 32;
  const int cap = model == CLOSURE_MLP ? 2 * sm_count() : 8 * sm_count();
  const int blocks = (int)std::min<int64_t>((groups + kClWarps - 1) / kClWarps, cap);
  if (model == CLOSURE_MLP)
    k_les_closure<T, CLOSURE_MLP><<<blocks, kClWarps * 32, 0, s>>>(a);
  else
    k_les_closure<T, CLOSURE_SMAGORINSKY><<<blocks, kClWarps * 32, 0, s>>>(a);
  SNS_CHECK_LAUNCH("k_les_closure");
  return OK;
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
  int rc;
  auto pass = [&](int axis, int first, int count, int sign, int pro, bool from_v) -> int {
    FieldPtrs f{};
    f.n = count;
    f.first = first;
    for (int i = 0; i < count; i++) {
      f.out[i] = U[first + i];
      f.in[i] = from_v ? (i < 3 ? V[i] : nullptr) : U[first + i];
    }
    LineGeo g = axis_geo(axis, nx, ny, nz, prec, pl.lineW);
    return run_line_pass(g, f, sign, 0, 1.0, prec, s, pro);
  };
  // inverse of V (3) and grad V (9): z with the gradient prologue, then y, x
  if ((rc = pass(2, 0, kLESWork, +1, PRO_GRAD12, true))) return rc;
  for (int axis : {1, 0})
    if ((rc = pass(axis, 0, kLESWork, +1, PRO_LOAD, false))) return rc;
  // pointwise closure
  {
    ClosureArgs a{};
    for (int q = 0; q < kLESWork; q++) a.U[q] = U[q];
    a.n = n;
    a.invN = 1.0 / (double)n;
    a.csd2 = cl.csd2;
    a.mlp = reinterpret_cast<const MlpPacked*>(cl.mlp);
    rc = prec == PREC_C128 ? launch_closure<double>(a, cl.model, s)
                           : launch_closure<float>(a, cl.model, s);
    if (rc) return rc;
  }
  // forward x, y of u x omega (U[0..2]) and tau (U[3..8]); z of tau
  for (int axis : {0, 1})
    if ((rc = pass(axis, 0, 9, -1, PRO_LOAD, false))) return rc;
  if ((rc = pass(2, 3, 6, -1, PRO_LOAD, false))) return rc;
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
  a.W = pl.zW;
  a.hK = dt / 2;
  a.nuhK = nu * dt / 2;
  a.stats = stats;
  a.kc2 = pl.kc2;
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
