// Vector::cross for callers that cannot allocate device memory.
//
// sns_cross takes its six work fields from the library's caching pool, which
// calls cudaMalloc the first time a size is seen.  Some callers cannot let
// that happen: a process whose device memory is already fully reserved by
// another allocator (a framework's caching allocator holding the whole GPU,
// or a fixed memory budget per process), or a loop that must never take the
// driver's allocation path at an unpredictable moment.  For them,
// sns_cross_noalloc runs the same kernels on a work area that is part of the
// library image itself: a file-scope __device__ array, created once per GPU
// when this file's code is first used and kept until the process exits.
//
// Because that array is a single static object, every call on a device uses
// the same bytes: calls that run at the same time on the GPU (on different
// streams) race with each other and must be serialised by the caller.  Each
// call rewrites the whole part of the array it reads (work fields and
// twiddle tables), so nothing carries over from one call to the next.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

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

// Device address of g_cross_scratch on the current device.  The host-side
// name of a __device__ array is only a stand-in, so the address is looked up
// once per device (with that device current) and cached.
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
    if (e != cudaSuccess)
      return sns::cuda_status(e, "sns_cross_noalloc: cudaGetSymbolAddress");
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
  if (prec != SNS_C64 && prec != SNS_C128) {
    set_error("sns_cross_noalloc: precision must be SNS_C64 or SNS_C128");
    return ERR_ARG;
  }
  if (!a || !b || !out) {
    set_error("sns_cross_noalloc: null vector");
    return ERR_ARG;
  }
  for (int d = 0; d < 3; d++)
    if (!a[d] || !b[d] || !out[d]) {
      set_error("sns_cross_noalloc: null field pointer");
      return ERR_ARG;
    }
  if (nx < 1 || ny < 1 || nz < 1 || !line_supported(nx) || !line_supported(ny) ||
      !line_supported(nz)) {
    set_error("sns_cross_noalloc: dimensions must be powers of two up to 4096");
    return ERR_ARG;
  }
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
  // twiddle tables of the three axes, written into the static area
  const void* tw[3] = {nullptr, nullptr, nullptr};
  const int64_t dims[3] = {nx, ny, nz};
  for (int ax = 0; ax < 3; ax++) {
    if (dims[ax] < 2) continue;
    std::vector<unsigned char> table;
    twiddle_host_table((int)dims[ax], prec, table);
    unsigned char* slot = base + kWorkBytes + ax * kTwiddleSlot;
    cudaError_t e = cudaMemcpyAsync(slot, table.data(), table.size(), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_status(e, "sns_cross_noalloc: twiddle upload");
    tw[ax] = slot;
  }
  const Dims d{(int)nx, (int)ny, (int)nz};
  return vector_cross(a, b, out, d, prec, work, s, tw);
}
