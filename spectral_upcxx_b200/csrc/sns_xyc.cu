// The xy phase of the fused NS step -- K2 (y-inverse of u and omega), K3 (x
// cross pass) and K4 (y-forward of the product) -- as one pass over each xy
// plane on a thread-block cluster (src/Vector.cpp:66-90 for one z plane: the
// y and x phases of Scalar::transform, src/Scalar.cpp:419-566, around the
// complex point-wise u x omega).
//
// For nx = ny = L (128 or 256) a cluster of CL = L/16 CTAs owns one plane at a
// time; CTA r of the cluster owns columns x in [16 r, 16 r + 16) in the y
// phases and rows y in [16 r, 16 r + 16) in the x phase.  Per plane:
//
//   1. y-inverse of the six fields on the CTA's 16 columns: straight from HBM
//      into registers (a half-warp reads 16 adjacent x, 128 bytes), the line
//      FFT's exchange in a column-interleaved scratch, and each result element
//      stored into the shared memory of the CTA that owns its row
//      (st.shared::cluster), so the six row blocks (6 x 16 rows) assemble in
//      the row owners without touching HBM;
//   2. cluster barrier; x-inverse of the 96 rows in place, the 1/N^2-scaled
//      complex cross product u x omega into the u rows, x-forward of the three
//      product rows in place;
//   3. cluster barrier (every CTA is done with its omega rows); each product
//      element stored into the omega region of the CTA that owns its column,
//      column-interleaved; cluster barrier;
//   4. y-forward of the three products on the CTA's columns, in place, and the
//      store to HBM (128-byte runs).
//
// HBM traffic of the phase: the six fields read once and the three products
// written once (9 field-passes instead of the 27 of three separate passes).
// Rows use an XOR swizzle within each group of 16 positions, and the column
// blocks interleave the 16 columns, so that every access of a half-warp --
// the line FFTs' loads and stage writes, the cross product, and the remote
// stores -- falls on 16 distinct 8-byte slots.  Arithmetic is that of the
// separate passes (same line FFT, same twiddle tables, same cross-product
// expression), so both give the same step.
//
// Measured on B200 (complex64): the pass is bound by the latency of its
// serial phases, not by HBM.  At 256^3 seven 16-CTA clusters are resident
// (112 SMs at one CTA each, 224 KB of shared memory) and one plane takes
// 39 us whether one cluster or seven run: y-inverse of the six fields with
// the stores to the row owners 15 us, x-inverse 7.2, x-forward 3.7, y-forward
// 3.5, product exchange 2.9, cross product 1.4, the four cluster barriers
// 3.6 us.  The phase takes 1.28 ms against 0.73 ms for the three separate
// passes (0.158 against 0.109 ms at 128^3), so the stepper uses the separate
// passes and this pass is opt-in (SNS_XYC=1).
#include <stdlib.h>

#include "sns_cluster.cuh"
#include "sns_common.cuh"
#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_tiles.cuh"
#include "sns_xy.cuh"

namespace sns {
namespace {

constexpr int kXYCThreads = 512;
constexpr int kXYCR = 16;  // rows (and columns) of a plane per CTA
constexpr size_t kSmemOptin = 232448;  // B200: 227 KB of dynamic shared memory per CTA

template <int L>
__host__ __device__ constexpr int xyc_cluster() {
  return L / kXYCR;
}

// Threads of the y lines of one field on the CTA's 16 columns, and how many
// such groups the CTA holds.
template <int L>
__host__ __device__ constexpr int xyc_group() {
  return kXYCR * LinePlan<L>::TPL;
}
template <int L>
__host__ __device__ constexpr int xyc_groups() {
  return kXYCThreads / xyc_group<L>();
}

// Elements of one field's 16-row (or 16-column) slice of a plane.
template <int L>
__host__ __device__ constexpr int xyc_slice() {
  return kXYCR * L;
}

// y-inverse scratch buffers: one per group when shared memory allows, else
// the groups take turns.
template <typename T, int L>
__host__ __device__ constexpr int xyc_scratch_buffers() {
  int n = xyc_groups<L>();
  while (n > 1 && (size_t)(6 + n) * xyc_slice<L>() * sizeof(cx_t<T>) > kSmemOptin) n /= 2;
  return n;
}

template <typename T, int L>
__host__ __device__ constexpr size_t xyc_smem_bytes() {
  return (size_t)(6 + xyc_scratch_buffers<T, L>()) * xyc_slice<L>() * sizeof(cx_t<T>);
}

// Slot of position p of row r in a row block: the low four bits of p are
// XORed with the group index p / 16 (and, where two lines share a half-warp,
// with 8 times the row's parity), which spreads the 16 lanes of every x-line
// access pattern over 16 distinct slots.
template <int L>
__device__ __forceinline__ int row_slot(int p, int r) {
  constexpr int LH = 16 / LinePlan<L>::TPL;  // lines per half-warp in the x phase
  return p ^ (((p >> 4) ^ ((r % LH) * (16 / LH))) & 15);
}

// blockIdx.x = cluster * CL + rank; cluster c takes the planes c, c + clusters, ...
template <typename T, int L>
__global__ void __launch_bounds__(kXYCThreads, 1)
    k_xy_cross(const FieldPtrs f, int nz, const cx_t<T>* __restrict__ tw, T scale2) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL, R = kXYCR;
  constexpr int GT = xyc_group<L>(), NG = xyc_groups<L>();
  constexpr int NYS = xyc_scratch_buffers<T, L>();
  constexpr int FL = xyc_slice<L>();
  constexpr int LPR = kXYCThreads / TPL;  // x lines per round
  static_assert(TPL <= 16 && kXYCThreads % GT == 0 && NG % NYS == 0, "cluster xy geometry");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* rb = reinterpret_cast<C*>(smem_raw);  // 6 fields x R rows x L, swizzled rows
  C* ys = rb + 6 * FL;                      // NYS scratch slices, column-interleaved
  const uint32_t rb_s = (uint32_t)__cvta_generic_to_shared(rb);
  const int rank = (int)cluster_rank();
  const int cid = (int)cluster_id_x(), ncl = (int)cluster_count_x();
  const int t = threadIdx.x;
  const int grp = t / GT, tl = t - grp * GT;
  const int w = tl % R, j = tl / R;  // y lines: column x0 + w, thread j of the line
  const int x0 = rank * R;
  const int lj = t % TPL, lline = t / TPL;  // x lines: thread lj of line lline of a round
  const int64_t plane = (int64_t)L * L;
  auto gsync = [grp] { named_bar(1 + grp, GT); };
  auto wsync = [] { line_sync<TPL>(); };
  auto col = [w](int p) { return p * R + w; };

  for (int z = cid; z < nz; z += ncl) {
    // every CTA of the cluster is done with its shared memory of the last plane
    cluster_sync();
    // ---- 1. y-inverse of the six fields; each element to the owner of its row
#pragma unroll 1
    for (int k = 0; k < (6 + NG - 1) / NG; k++) {
      const int fld = grp + NG * k;
      const bool act = fld < 6;
      C v[E];
      if (act) {
        const C* __restrict__ src =
            reinterpret_cast<const C*>(select_ptr(f.in, fld)) + z * plane + x0 + w;
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = src[(int64_t)(j + TPL * e) * L];
      }
#pragma unroll 1
      for (int turn = 0; turn < NG / NYS; turn++) {
        if (act && grp / NYS == turn)
          line_fft_at<L>(v, ys + (grp % NYS) * FL, col, j, tw, (T)1, gsync);
        if (NG / NYS > 1) __syncthreads();
      }
      if (act) {
#pragma unroll
        for (int e = 0; e < E; e++) {
          const int y = j + TPL * e, q = y / R, ly = y - q * R;
          const int slot = (fld * R + ly) * L + row_slot<L>(x0 + w, ly);
          st_cluster(cluster_addr(rb_s + (uint32_t)(slot * (int)sizeof(C)), (uint32_t)q), v[e]);
        }
      }
    }
    cluster_sync();
    // ---- 2. x-inverse of the 6 R rows, cross product, x-forward of the 3 R product rows
#pragma unroll 1
    for (int l0 = 0; l0 < 6 * R; l0 += LPR) {
      const int li = l0 + lline;
      if (li < 6 * R) {
        const int r = li % R;
        C* row = rb + li * L;
        auto rs = [r](int p) { return row_slot<L>(p, r); };
        C v[E];
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = row[rs(lj + TPL * e)];
        wsync();
        line_fft_at<L>(v, row, rs, lj, tw, (T)1, wsync);
#pragma unroll
        for (int e = 0; e < E; e++) row[rs(lj + TPL * e)] = v[e];
      }
    }
    __syncthreads();
    // c = (u/N) x (omega/N) (src/Vector.cpp:79-84), as the separate x pass forms it
#pragma unroll 1
    for (int q = t; q < FL; q += kXYCThreads) {
      const int r = q / L, p = q - r * L;
      const int s = r * L + row_slot<L>(p, r);
      C u[3], o[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        u[d] = rb[d * FL + s];
        o[d] = rb[(3 + d) * FL + s];
      }
      const C c0 = csub(cmul(u[1], o[2]), cmul(u[2], o[1]));
      const C c1 = csub(cmul(u[2], o[0]), cmul(u[0], o[2]));
      const C c2 = csub(cmul(u[0], o[1]), cmul(u[1], o[0]));
      rb[0 * FL + s] = cscale(scale2, c0);
      rb[1 * FL + s] = cscale(scale2, c1);
      rb[2 * FL + s] = cscale(scale2, c2);
    }
    // this CTA has read its omega rows: they may receive the product columns
    cluster_arrive();
    __syncthreads();
#pragma unroll 1
    for (int l0 = 0; l0 < 3 * R; l0 += LPR) {
      const int li = l0 + lline;
      if (li < 3 * R) {
        const int r = li % R;
        C* row = rb + li * L;
        auto rs = [r](int p) { return row_slot<L>(p, r); };
        C v[E];
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = row[rs(lj + TPL * e)];
        wsync();
        line_fft_at<L>(v, row, rs, lj, tw, (T)-1, wsync);
#pragma unroll
        for (int e = 0; e < E; e++) row[rs(lj + TPL * e)] = v[e];
      }
    }
    __syncthreads();
    cluster_wait();
    // ---- 3. product rows to the column owners (omega region, column-interleaved)
#pragma unroll 1
    for (int q = t; q < 3 * FL; q += kXYCThreads) {
      const int fld = q / FL, rem = q - fld * FL;
      const int r = rem / L, p = rem - r * L;
      const C val = rb[fld * FL + r * L + row_slot<L>(p, r)];
      const int owner = p / R, wc = p - owner * R;
      const int slot = (3 + fld) * FL + (x0 + r) * R + wc;
      st_cluster(cluster_addr(rb_s + (uint32_t)(slot * (int)sizeof(C)), (uint32_t)owner), val);
    }
    cluster_sync();
    // ---- 4. y-forward of the three products on this CTA's columns, to HBM
#pragma unroll 1
    for (int k = 0; k < (3 + NG - 1) / NG; k++) {
      const int fld = grp + NG * k;
      if (fld < 3) {
        C* cb = rb + (3 + fld) * FL;
        C v[E];
#pragma unroll
        for (int e = 0; e < E; e++) v[e] = cb[col(j + TPL * e)];
        gsync();
        line_fft_at<L>(v, cb, col, j, tw, (T)-1, gsync);
        C* __restrict__ dst = reinterpret_cast<C*>(select_ptr(f.out, fld)) + z * plane + x0 + w;
#pragma unroll
        for (int e = 0; e < E; e++) dst[(int64_t)(j + TPL * e) * L] = v[e];
      }
    }
  }
}

template <typename T, int L>
cudaLaunchConfig_t xyc_config(cudaLaunchAttribute* at, int clusters, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(xyc_cluster<L>() * clusters));
  cfg.blockDim = dim3(kXYCThreads);
  cfg.dynamicSmemBytes = xyc_smem_bytes<T, L>();
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = xyc_cluster<L>();
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

// Clusters of k_xy_cross<T, L> that the device runs at once (0: none fits),
// asked once per device; the kernel attributes are set on the way.
template <typename T, int L>
int xyc_clusters_resident() {
  static int known[64];
  static bool asked[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!asked[dev & 63]) {
    int n = 0;
    cudaError_t e = cudaFuncSetAttribute(k_xy_cross<T, L>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)xyc_smem_bytes<T, L>());
    if (e == cudaSuccess && xyc_cluster<L>() > 8)
      e = cudaFuncSetAttribute(k_xy_cross<T, L>, cudaFuncAttributeNonPortableClusterSizeAllowed,
                               1);
    if (e == cudaSuccess) {
      cudaLaunchAttribute at[1];
      cudaLaunchConfig_t cfg = xyc_config<T, L>(at, 1, nullptr);
      e = cudaOccupancyMaxActiveClusters(&n, k_xy_cross<T, L>, &cfg);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();  // a refused query leaves no error behind
      n = 0;
    }
    known[dev & 63] = n;
    asked[dev & 63] = true;
  }
  return known[dev & 63];
}

template <typename T, int L>
int launch_xyc(void* const U[6], int nz, double scale2, cudaStream_t s) {
  using C = cx_t<T>;
  const int resident = xyc_clusters_resident<T, L>();
  if (resident <= 0) {
    set_error("cluster xy pass: no cluster fits on this device");
    return ERR_UNSUPPORTED;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  FieldPtrs f{};
  f.n = 6;
  for (int i = 0; i < 6; i++) f.in[i] = U[i];
  for (int i = 0; i < 3; i++) f.out[i] = U[i];
  const int clusters = nz < resident ? nz : resident;
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg = xyc_config<T, L>(at, clusters, s);
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_xy_cross<T, L>, f, nz, tw, (T)scale2);
  if (e != cudaSuccess) return cuda_status(e, "k_xy_cross");
  return OK;
}

}  // namespace

bool xyc_supported(int nx, int ny, int prec) {
  const char* env = getenv("SNS_XYC");
  if (!(env && env[0] == '1')) return false;
  if (nx != ny) return false;
  if (nx == 128)
    return prec == PREC_C128 ? xyc_clusters_resident<double, 128>() > 0
                             : xyc_clusters_resident<float, 128>() > 0;
  if (nx == 256 && prec == PREC_C64) return xyc_clusters_resident<float, 256>() > 0;
  return false;
}

int xyc_run(void* const U[6], int nx, int ny, int nz, int prec, cudaStream_t s) {
  const double N = (double)nx * ny * nz;
  const double scale2 = 1.0 / (N * N);
  if (nx == ny && nx == 128)
    return prec == PREC_C128 ? launch_xyc<double, 128>(U, nz, scale2, s)
                             : launch_xyc<float, 128>(U, nz, scale2, s);
  if (nx == ny && nx == 256 && prec == PREC_C64) return launch_xyc<float, 256>(U, nz, scale2, s);
  set_error("cluster xy pass: nx = ny = 128, or 256 in complex64");
  return ERR_UNSUPPORTED;
}

}  // namespace sns
