// Batched line-FFT passes over device fields (host interface).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include <stddef.h>

#include "sns_common.cuh"

namespace sns {

constexpr int kMaxFields = 12;
constexpr int kMaxLine = 4096;

// cos and sin of 2 pi m / n in FP64, with the angle reduced to the first
// octant so that the FP64 sine and cosine see |t| <= pi/4.  The host twiddle
// tables and the on-device tables of the allocation-free entry point use it.
__host__ __device__ inline void cis_octant(int64_t m, int64_t n, double* c, double* s) {
  m %= n;
  if (m < 0) m += n;
  const int64_t m8 = 8 * m;
  const int64_t oct = m8 / n;
  const int64_t rem = m8 - oct * n;
  const double t = (oct & 1) ? (M_PI / 4) * ((double)(n - rem) / (double)n)
                             : (M_PI / 4) * ((double)rem / (double)n);
  const double ct = cos(t), st = sin(t);
  double x, y;
  switch (oct) {
    case 0: x = ct; y = st; break;
    case 1: x = st; y = ct; break;
    case 2: x = -st; y = ct; break;
    case 3: x = -ct; y = st; break;
    case 4: x = -ct; y = -st; break;
    case 5: x = -st; y = -ct; break;
    case 6: x = st; y = -ct; break;
    default: x = ct; y = -st; break;
  }
  *c = x;
  *s = y;
}

// Epilogue flags of a pass.
enum PassFlags : int {
  PASS_SCALE = 1,         // multiply the output by `scale`
  PASS_ZERO_NYQUIST = 2,  // zero outputs on the planes x=nx/2, y=ny/2, z=nz/2
};

// How a pass forms its input tile.
enum PassPrologue : int {
  PRO_LOAD = 0,   // field f reads in[f]
  PRO_CURL6 = 1,  // in[0..2] = a Fourier vector V; fields 0..2 read V, fields
                  // 3..5 form (i k x V) on the fly (src/Vector.cpp:92-122)
  PRO_IKAXIS = 3,  // field f reads in[f], times i k (the wavenumber along the
                   // line) when bit f of ikmask is set: a derivative along the
                   // pass axis taken on the way in
  PRO_OMEGA = 4,   // y lines after a z pass: in[0..2] = the z-inverted V,
                   // in[3..4] = the z-inverted i kz Vx, i kz Vy; fields 0..2
                   // read V, fields 3..5 form omega = i k x V from them
                   // (i ky Vz - dzVy, dzVx - i kx Vz, i kx Vy - i ky Vx)
};

// Geometry of a batch of lines: element p of line (w, g) of tile t sits at
//   base(t) + w + g*gs + p*ps,  base(t) = (t % TA)*sa + (t / TA)*sb.
// W adjacent lines (unit stride) and G line groups form one tile.
struct LineGeo {
  int L;       // line length (power of two)
  int W, G;    // adjacent lines and groups per tile
  int64_t ps, gs;
  int64_t TA, TB, sa, sb;
  // field dimensions and the axis of the lines (0, 1, 2; -1 for plain 1D
  // batches), used by the curl prologue and the Nyquist epilogue
  int nx, ny, nz;
  int axis;
  // twiddle table to use instead of the cached one (null: cached table)
  const void* tw;
  // half-spectrum fields of a real-field run: x index i holds kx = i
  // (0 <= i < nx), the kx < 0 half being the complex conjugate; no x-Nyquist
  int kx_half;
  // radix order of the line FFT (RadixOrder; plain-load passes of 64..1024)
  int ord;
  // L2 prefetch: each CTA asks L2 for the inputs of the tile pf launches
  // ahead (0: none); the launcher sets pf to pfw waves of resident CTAs
  int64_t pf;
  int pfw;
};

// Tiles in `waves` waves of a kernel's resident CTAs on this device.
template <typename K>
inline int64_t tiles_in_waves(K* kernel, int threads, size_t smem, int waves) {
  if (waves <= 0) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return (int64_t)waves * per_sm * sm_count();
}

struct FieldPtrs {
  void* in[kMaxFields];
  void* out[kMaxFields];
  int n;
  unsigned ikmask;  // PRO_IKAXIS: fields whose input is multiplied by i k_axis
};

bool is_pow2(int64_t n);
// Validate that the batched pass supports line length L.
bool line_supported(int64_t L);

// One transform pass along the lines of `geo` over `f.n` fields.
// sign = -1 forward, +1 inverse.  In place when in == out.
int run_line_pass(const LineGeo& geo, const FieldPtrs& f, int sign, int flags, double scale,
                  int prec, cudaStream_t stream, int prologue = PRO_LOAD);

// The same pass (plain loads only, x, y or z lines, 1..6 fields, L = 32..512;
// x lines of at most 256 8-byte units)
// as a persistent pass over TMA-staged tiles with `stages` (1 or 2) shared
// memory stages (sns_line_tma.cu); its bounded waits record into *err
// (1: a wait ran out, 2: a box failed the kernel's own check).  Same results
// bit for bit as run_line_pass.
bool line_tma_ok(const LineGeo& geo, int prec, int stages);
int run_line_pass_tma(const LineGeo& geo, const FieldPtrs& f, int sign, int flags, double scale,
                      int prec, cudaStream_t stream, int stages, int* err);

// Geometry of the lines along `axis` (0 = x, 1 = y, 2 = z) of nx*ny*nz fields.
// wmax > 0 caps the adjacent lines per tile at that width (a tuned value).
// Geometry of the lines along `axis`; wmax caps the adjacent lines of a tile,
// tmax the threads up to which line groups are added (0: defaults), ord is
// the radix order (RadixOrder).
LineGeo axis_geo(int axis, int nx, int ny, int nz, int prec, int wmax = 0, int tmax = 0,
                 int ord = 0);

// Full 3D C2C transform of nf fields in place (the Scalar::transform
// contract, src/Scalar.cpp:400-646), with optional fused Nyquist zeroing
// (forward) and 1/N scaling (inverse).
// tw_axes, when given, holds the twiddle table of each axis (x, y, z) to use
// instead of the cached tables.
// x and y axes in one pass over each xy plane (thread-block clusters with
// distributed shared memory, sns_fft_xy.cu): fft3d uses it where nx = ny =
// 128 (measured faster there); SNS_FFT_XY=0 keeps the three line passes.
bool fft_xy_supported(int nx, int ny, int nz, int nf, int prec);
int fft_xy_pass(const FieldPtrs& f, int nx, int nz, int sign, int flags, double scale, int prec,
                cudaStream_t s);
int fft3d(void* const* fields, int nf, int nx, int ny, int nz, int sign, int flags,
          int prec, cudaStream_t stream, const void* const* tw_axes = nullptr);

// Tuned plan of a 3D transform shape: per axis the tile knobs of axis_geo,
// and whether the xy plane pass is used where it is available.
struct FftChoice {
  int wmax[3], tmax[3], ord[3];
  int tma[3];  // stages of the TMA-staged form of each axis's pass (0: direct loads)
  bool plane;
};
// Error word of the transform's TMA-staged passes on the current device
// (null if it cannot be set up), and its check: reads and clears it,
// SNS_ERR_TIMEOUT with the error text when a pass recorded a failure.
int* fft_tma_err_word();
int fft_tma_check(cudaStream_t s);
// Measure candidate plans for nf fields of nx*ny*nz on pool scratch fields and
// cache the fastest for this device (the counterpart of FFTW_MEASURE,
// src/FFT1D.cpp:18-22); fft3d then uses it for that shape.
int fft3d_tune(int nx, int ny, int nz, int nf, int prec, cudaStream_t stream);
// The cached choice of a shape, if any (no tuning).
bool fft3d_tuned(int nx, int ny, int nz, int nf, int prec, FftChoice* out);
// SNS_TUNE=1: transforms and steppers tune each new shape on first use.
bool tune_on_first_use();

// Device twiddle table exp(-2 pi i m / L), m < L, generated in FP64 on the
// host and stored as complex64 or complex128 (cached per device).
const void* twiddles(int L, int prec);
// The same table as host bytes (L complex values of the precision).
void twiddle_host_table(int L, int prec, std::vector<unsigned char>& out);

}  // namespace sns
