// x and y axes of a 3D FFT in one pass over each xy plane, for nx = ny = L
// in {128, 256}: a thread-block cluster of CL CTAs (16 at L = 256, 8 at 128)
// holds one plane in its distributed shared memory.  CTA r of the cluster
//   1. loads rows y in [r R, r R + R) of the plane (R = L / CL), transforms
//      them along x and keeps them in its shared memory;
//   2. after a cluster barrier, gathers columns x in [r R, r R + R) -- each
//      column's L values from the CTAs that own its rows -- into registers
//      through distributed shared memory (mapa + ld.shared::cluster);
//   3. after a second cluster barrier (every CTA has read what it needs, so
//      its own shared memory is free), transforms the columns along y with
//      its shared memory as exchange space and writes them back.
// The plane crosses HBM once per direction instead of twice (x pass + y
// pass), so a 3D transform is two passes (xy planes + z lines) instead of
// three (src/Scalar.cpp:400-646 runs y, x, z).  The epilogue (1/N, Nyquist
// zeroing) rides on whichever pass is last, as in the three-pass path.
// Measured on B200: at 128^3 complex64 a forward + inverse pair takes 55 us
// against 62 us in three passes, so fft3d uses it there; at 256^3 the pass
// is latency-bound (each cluster loads, exchanges and stores one plane with
// two cluster barriers and nothing to overlap them: 403 us against 325 us)
// and fft3d keeps the line passes.
#include "../../include/spectral_b200.h"
#include "sns_cluster.cuh"
#include "sns_common.cuh"
#include "sns_fft.cuh"
#include "sns_fft_core.cuh"
#include "sns_tiles.cuh"

namespace sns {
namespace {

// CTAs per cluster: 8 at L = 128; 16 at L = 256 (a non-portable cluster
// size: CTAs of 16 rows, two per SM), the measured variant
template <int L>
__host__ __device__ constexpr int xy_cluster() {
  return L == 256 ? 16 : 8;
}

template <int L>
__host__ __device__ constexpr int xy_threads() {
  return (L / xy_cluster<L>()) * LinePlan<L>::TPL;
}

template <typename T, int L>
constexpr size_t xy_smem_bytes() {
  constexpr int R = L / xy_cluster<L>();
  constexpr int es = (int)sizeof(cx_t<T>);
  constexpr int a = R * xrow_stride(L, es), b = R * tile_stride(L, R, es);
  return (size_t)(a > b ? a : b) * sizeof(cx_t<T>);
}

// blockIdx.x: rank in the cluster; blockIdx.y: field * nz + z
template <typename T, int L>
__global__ void __launch_bounds__(xy_threads<L>(), 2)
    k_fft_xy(const FieldPtrs f, int nz, const cx_t<T>* __restrict__ tw, T sg, T scale,
             int flags) {
  using C = cx_t<T>;
  using P = LinePlan<L>;
  constexpr int E = P::E, TPL = P::TPL, R = L / xy_cluster<L>();
  constexpr int RSX = xrow_stride(L, (int)sizeof(C)), RSY = tile_stride(L, R, (int)sizeof(C));
  static_assert(TPL <= 32, "row lines stay within a warp");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sm = reinterpret_cast<C*>(smem_raw);
  const int rank = blockIdx.x;
  const int field = blockIdx.y / nz, z = blockIdx.y - field * nz;
  C* __restrict__ data = reinterpret_cast<C*>(select_ptr(f.out, field)) + (int64_t)z * L * L;
  const int t = threadIdx.x;
  // 1. rows: x lines, kept in shared memory in natural order
  {
    const int row = t / TPL, j = t % TPL;
    const C* __restrict__ src = data + (int64_t)(rank * R + row) * L + j;
    C v[E];
#pragma unroll
    for (int e = 0; e < E; e++) v[e] = src[TPL * e];
    C* r = sm + row * RSX;
    line_fft<L>(v, r, j, tw, sg);
#pragma unroll
    for (int e = 0; e < E; e++) r[pad_pos(j + TPL * e)] = v[e];
  }
  cluster_sync();
  // 2. columns: element y of column x lives in CTA y / R, row y % R
  const int c = t % R, j = t / R;
  const int x = rank * R + c;
  C v[E];
  {
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(sm);
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int y = j + TPL * e;
      const int q = y / R, ly = y - q * R;
      const uint32_t a = base + (uint32_t)((ly * RSX + pad_pos(x)) * (int)sizeof(C));
      v[e] = ld_cluster(cluster_addr(a, (uint32_t)q), (const C*)nullptr);
    }
  }
  cluster_sync();
  // 3. y lines of the R columns (thread index c fastest: block-synchronised stages)
  line_fft<L, true>(v, sm + c * RSY, j, tw, sg);
  const bool do_scale = flags & PASS_SCALE;
  const bool do_zero = flags & PASS_ZERO_NYQUIST;
  const bool on_plane = x == (L >> 1) || z == (nz >> 1);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int y = j + TPL * e;
    C val = v[e];
    if (do_scale) val = cscale(scale, val);
    if (do_zero && (on_plane || y == (L >> 1))) val = mk((T)0, (T)0);
    data[(int64_t)y * L + x] = val;
  }
}

template <typename T, int L>
int launch_xy(const FieldPtrs& f, int nz, int sign, int flags, double scale, cudaStream_t s) {
  using C = cx_t<T>;
  constexpr size_t smem = xy_smem_bytes<T, L>();
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(k_fft_xy<T, L>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && xy_cluster<L>() > 8)
      e = cudaFuncSetAttribute(k_fft_xy<T, L>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(k_fft_xy)");
    attr[dev & 63] = true;
  }
  const C* tw = reinterpret_cast<const C*>(twiddles(L, sizeof(T) == 8 ? PREC_C128 : PREC_C64));
  if (!tw) {
    set_error("twiddle table allocation failed");
    return ERR_ALLOC;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(xy_cluster<L>(), (unsigned)(nz * f.n));
  cfg.blockDim = dim3(xy_threads<L>());
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = xy_cluster<L>();
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, k_fft_xy<T, L>, f, nz, tw, (T)sign, (T)scale, flags);
  if (e != cudaSuccess) return cuda_status(e, "k_fft_xy");
  return OK;
}

}  // namespace

namespace {

// Whether a cluster of the plane pass fits on this device (for example not
// under a partition too small for an 8-CTA cluster): asked once per device
// and precision.
template <typename T, int L>
bool clusters_fit() {
  static int known[64] = {0};  // 0: not asked, 1: fits, 2: does not
  int dev = 0;
  cudaGetDevice(&dev);
  if (!known[dev & 63]) {
    constexpr size_t smem = xy_smem_bytes<T, L>();
    int n = 0;
    cudaError_t e = cudaFuncSetAttribute(k_fft_xy<T, L>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(xy_cluster<L>(), 1);
      cfg.blockDim = dim3(xy_threads<L>());
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = xy_cluster<L>();
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      e = cudaOccupancyMaxActiveClusters(&n, k_fft_xy<T, L>, &cfg);
    }
    if (e != cudaSuccess) cudaGetLastError();  // a refused query leaves no error behind
    known[dev & 63] = (e == cudaSuccess && n > 0) ? 1 : 2;
  }
  return known[dev & 63] == 1;
}

}  // namespace

bool fft_xy_supported(int nx, int ny, int nz, int nf, int prec) {
  const char* env = getenv("SNS_FFT_XY");
  if (env && env[0] == '0') return false;
  if (!(nx == ny && nx == 128 && nz >= 1 && (int64_t)nz * nf <= 65535)) return false;
  return prec == PREC_C128 ? clusters_fit<double, 128>() : clusters_fit<float, 128>();
}

int fft_xy_pass(const FieldPtrs& f, int nx, int nz, int sign, int flags, double scale, int prec,
                cudaStream_t s) {
  if (nx == 128)
    return prec == PREC_C128 ? launch_xy<double, 128>(f, nz, sign, flags, scale, s)
                             : launch_xy<float, 128>(f, nz, sign, flags, scale, s);
  set_error("xy plane pass: nx = ny = 128");
  return ERR_UNSUPPORTED;
}

}  // namespace sns
