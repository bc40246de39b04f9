// Shared device helpers: complex types, error plumbing, grid sizing.
#pragma once

#include <stdlib.h>

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace sns {

// Precision codes of the C-ABI (spectral_b200.h): 0 = complex64, 1 = complex128.
enum Prec : int { PREC_C64 = 0, PREC_C128 = 1 };

template <typename T>
struct cx;
template <>
struct cx<float> {
  using type = float2;
};
template <>
struct cx<double> {
  using type = double2;
};
template <typename T>
using cx_t = typename cx<T>::type;

__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <typename C>
__device__ __forceinline__ C cadd(C a, C b) {
  return mk(a.x + b.x, a.y + b.y);
}
template <typename C>
__device__ __forceinline__ C csub(C a, C b) {
  return mk(a.x - b.x, a.y - b.y);
}
template <typename C>
__device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// (0, k) * z, the product std::complex forms for i*k*z.
template <typename C, typename T>
__device__ __forceinline__ C ikmul(T k, C z) {
  return mk(-k * z.y, k * z.x);
}
template <typename C, typename T>
__device__ __forceinline__ C cscale(T s, C z) {
  return mk(s * z.x, s * z.y);
}

// Largest CTA of the FFT kernels: FP64 lines need about twice the registers.
template <typename T>
struct MaxThreads {
  static constexpr int value = sizeof(T) == 8 ? 512 : 768;
};
inline int max_threads(int prec) { return prec == PREC_C128 ? 512 : 768; }

// Scalar::freq (src/Scalar.cpp:198-206): k = i for i <= n/2, else i - n.
__device__ __forceinline__ int freq_i(int i, int n) { return (i <= (n >> 1)) ? i : i - n; }

// Thread-local last-error string of the C-ABI.
void set_error(const std::string& msg);
const char* last_error();

// Status codes of the C-ABI.
enum Status : int {
  OK = 0,
  ERR_ARG = -1,
  ERR_UNSUPPORTED = -2,
  ERR_CUDA = -3,
  ERR_ALLOC = -4,
  ERR_TIMEOUT = -5,
};

int cuda_status(cudaError_t e, const char* where);

// Argument checks shared by the C-ABI entry points; each sets the error text
// and returns false on a bad argument.
bool check_prec(int prec);
bool check_dims(int64_t nx, int64_t ny, int64_t nz);
bool nonnull(const void* p, const char* what);
bool vec_ok(const void* const v[3], const char* what);

// Opt a kernel into the largest dynamic shared memory that its static shared
// memory leaves on this device.
template <typename K>
inline cudaError_t allow_max_dynamic_smem(K* kernel) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, (const void*)kernel);
  if (e != cudaSuccess) return e;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - (int)a.sharedSizeBytes);
}

// Number of SMs of the current device (cached).
int sm_count();

}  // namespace sns

// Programmatic dependent launch.  A kernel started by launch_pdl inside a
// PdlScope may begin while its predecessor in the stream is still draining:
// it first lets its own dependents be scheduled (pdl_trigger: they start once
// every CTA of this grid has started, so they never take an SM slot this grid
// still needs), then waits for the predecessor grid to complete with its
// memory visible (pdl_wait) before reading anything that grid wrote.  Both are
// no-ops after an ordinary launch.  Measured on B200: the 64^3 closure step
// gains 2.4 %, the 256^3 steps are unchanged and the 64^3 plain step loses
// 16 %, so only the closure step opens a scope.  SNS_PDL=0 turns it off.
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

inline bool& pdl_scope_flag() {
  static thread_local bool on = false;
  return on;
}
struct PdlScope {
  bool prev;
  PdlScope() : prev(pdl_scope_flag()) { pdl_scope_flag() = true; }
  ~PdlScope() { pdl_scope_flag() = prev; }
};
inline bool pdl_enabled() {
  static const bool allowed = [] {
    const char* e = getenv("SNS_PDL");
    return !(e && e[0] == '0');
  }();
  return allowed && pdl_scope_flag();
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                              cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

#define SNS_CHECK_LAUNCH(where)                                    \
  do {                                                             \
    cudaError_t _e = cudaGetLastError();                           \
    if (_e != cudaSuccess) return ::sns::cuda_status(_e, where);   \
  } while (0)
