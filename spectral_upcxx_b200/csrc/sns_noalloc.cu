// Vector::cross for callers that cannot allocate device memory.
//
// sns_cross takes its six work fields from the library's caching pool, which
// calls cudaMalloc the first time a size is seen, and its twiddle tables from
// a cache that does the same.  Some callers cannot let that happen: a process
// whose device memory is already fully reserved by another allocator (a
// framework's caching allocator holding the whole GPU, or a fixed memory
// budget per process), or a loop that must never take the driver's
// allocation path at an unpredictable moment.  For them, sns_cross_noalloc
// runs the same kernels on a work area that is part of the library image
// itself: a file-scope __device__ array, kept until the process exits.
//
// Set-up, once per device: the first call made with a device current looks
// up the array's device address with cudaGetSymbolAddress (the host-side name
// of a __device__ array is only a stand-in for it) and caches it.  Under the
// CUDA default of lazy module loading this lookup is also when the driver
// creates the array on that GPU, so it can fail with an out-of-memory error
// if another allocator has already taken the whole device: make the first
// call before that allocator reserves its memory (a warm-up call at start-up
// does it), and before any stream capture.
//
// Because the array is a single static object, every call on a device uses
// the same bytes, and the array keeps what the last call left there: calls
// that run at the same time on the GPU (on different streams) race with each
// other and must be serialised by the caller.  Each call rewrites every part
// of the array it reads -- the work fields and the twiddle tables, the latter
// generated by a kernel on the caller's stream -- so nothing carries over from
// one call to the next.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/spectral_b200.h"
#include "sns_common.cuh"
#include "sns_fft.cuh"
#include "sns_ops.cuh"

namespace {

// Six work fields of up to 2^18 complex128 values (64^3) -- 24 MiB -- plus one
// twiddle table per axis for lines of up to 4096 complex128 values.
constexpr size_t kWorkBytes = (size_t)6 * 262144 * 16;
constexpr size_t kTwiddleSlot = (size_t)sns::kMaxLine * 16;
constexpr size_t kScratchBytes = kWorkBytes + 3 * kTwiddleSlot;

static __device__ __align__(256) unsigned char g_cross_scratch[kScratchBytes];

// Twiddle table tw[m] = exp(-2 pi i m / L), m < L, computed in FP64 and
// rounded to T: the values of the host-generated tables of the pooled path
// (the same octant reduction; the device's FP64 sine and cosine in place of
// the host's).
template <typename T>
__global__ void k_twiddle_table(T* __restrict__ out, int L) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= L) return;
  double c, s;
  sns::cis_octant(m, L, &c, &s);
  out[2 * m] = (T)c;
  out[2 * m + 1] = (T)(-s);
}

// Device address of g_cross_scratch on the current device, looked up once per
// device with that device current and cached.
int scratch_address(unsigned char** out) {
  static std::mutex mu;
  static void* addr[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sns::cuda_status(e, "sns_cross_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 64) {
    sns::set_error("sns_cross_noalloc: device index out of range");
    return sns::ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_cross_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      sns::set_error(std::string("sns_cross_noalloc: the static work area (") +
                     std::to_string(kScratchBytes) +
                     " bytes) could not be set up on this device -- the first call must come "
                     "before another allocator reserves the device memory: " +
                     cudaGetErrorString(e));
      return sns::ERR_CUDA;
    }
    addr[dev] = p;
  }
  *out = static_cast<unsigned char*>(addr[dev]);
  return sns::OK;
}

}  // namespace

extern "C" int sns_cross_noalloc(const void* const a[3], const void* const b[3],
                                 void* const out[3], int64_t nx, int64_t ny, int64_t nz, int prec,
                                 void* stream) {
  using namespace sns;
  // the argument checks and return codes of sns_cross
  if (!check_prec(prec) || !check_dims(nx, ny, nz) || !vec_ok(a, "sns_cross_noalloc") ||
      !vec_ok(b, "sns_cross_noalloc") || !vec_ok((const void* const*)out, "sns_cross_noalloc"))
    return ERR_ARG;
  if (!line_supported(nx) || !line_supported(ny) || !line_supported(nz)) {
    set_error("sns_cross_noalloc: dimensions must be powers of two up to 4096");
    return ERR_UNSUPPORTED;
  }
  // the one limit of its own: the size of the static work area
  const size_t esz = prec == SNS_C128 ? 16 : 8;
  const size_t n = (size_t)nx * ny * nz;
  if (6 * n * esz > kWorkBytes) {
    set_error("sns_cross_noalloc: a " + std::to_string(nx) + "x" + std::to_string(ny) + "x" +
              std::to_string(nz) + " box needs " + std::to_string(6 * n * esz) +
              " bytes of work space; the static work area holds " +
              std::to_string(kWorkBytes) +
              " bytes (at most 262144 complex128 or 524288 complex64 points per field)");
    return ERR_ARG;
  }
  unsigned char* base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  void* work[6];
  for (int i = 0; i < 6; i++) work[i] = base + (size_t)i * n * esz;
  // twiddle tables of the three axes, generated into the static area
  const void* tw[3] = {nullptr, nullptr, nullptr};
  const int64_t dims[3] = {nx, ny, nz};
  for (int ax = 0; ax < 3; ax++) {
    if (dims[ax] < 2) continue;
    unsigned char* slot = base + kWorkBytes + ax * kTwiddleSlot;
    const int L = (int)dims[ax];
    const int threads = L < 256 ? L : 256;
    if (prec == SNS_C128)
      k_twiddle_table<double><<<(L + threads - 1) / threads, threads, 0, s>>>(
          reinterpret_cast<double*>(slot), L);
    else
      k_twiddle_table<float><<<(L + threads - 1) / threads, threads, 0, s>>>(
          reinterpret_cast<float*>(slot), L);
    SNS_CHECK_LAUNCH("sns_cross_noalloc: twiddle table");
    tw[ax] = slot;
  }
  const Dims d{(int)nx, (int)ny, (int)nz};
  return vector_cross(a, b, out, d, prec, work, s, tw);
}
