// FFT1D over the device line-FFT pass (sns_fft1d_many).  The reference runs
// one FFTW plan per strided line (src/FFT1D.cpp:14-101).  Here a line in
// device memory is transformed where it lies, strided, with no copy and no
// allocation; a line in host memory is staged through a device buffer that is
// kept between calls and grows to the longest line seen (the counterpart of
// the plan FFTW keeps), so repeated calls allocate nothing.  Work is queued on
// the legacy default stream, as for every field operation of this API; a host
// line is copied back before the call returns.
#include "FFT1D.H"

#include <cuda_runtime.h>

#include <iostream>

#include "sns_api_internal.H"

namespace {

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Device staging buffer for host lines, shared by all FFT1D objects of the
// process (one host thread calls the API, as in the reference).  It is held
// until the process exits, like the blocks of the field pool.
struct Staging {
  void* ptr = nullptr;
  size_t bytes = 0;
  void* get(size_t need) {
    if (need > bytes) {
      if (ptr) SNS_API_CHECK(sns_free(ptr));
      ptr = nullptr;
      SNS_API_CHECK(sns_malloc(&ptr, need));
      bytes = need;
    }
    return ptr;
  }
};
Staging g_staging;

void copy_failed() {
  std::cerr << "ERROR in FFT1D: line copy failed" << std::endl;
  std::exit(1);
}

// Transform one line of N elements `stride` apart in place; scale = 1 for the
// unnormalised transforms, 1/N for inverse().
void run_line(cdouble* input, int N, int stride, int dir, double scale) {
  if (N < 1 || stride < 1) {
    std::cerr << "ERROR in FFT1D: bad size or stride" << std::endl;
    std::exit(1);
  }
  if (is_device_pointer(input)) {
    SNS_API_CHECK(sns_fft1d_many_scaled(input, N, stride, 1, N, dir, scale, SNS_C128, nullptr));
    return;
  }
  const size_t esz = sizeof(cdouble);
  void* d = g_staging.get(esz * (size_t)N);
  // gather the (possibly strided) host line into the contiguous device buffer
  if (cudaMemcpy2DAsync(d, esz, input, esz * (size_t)stride, esz, N, cudaMemcpyHostToDevice,
                        nullptr) != cudaSuccess)
    copy_failed();
  SNS_API_CHECK(sns_fft1d_many_scaled(d, N, 1, 1, N, dir, scale, SNS_C128, nullptr));
  if (cudaMemcpy2DAsync(input, esz * (size_t)stride, d, esz, esz, N, cudaMemcpyDeviceToHost,
                        nullptr) != cudaSuccess)
    copy_failed();
  SNS_API_CHECK(sns_stream_synchronize(nullptr));
}

}  // namespace

FFT1D::FFT1D() : m_N(0), m_stride(1), m_dir(0), m_alignment(0) {}
FFT1D::~FFT1D() {}

void FFT1D::init(int N, int stride, cdouble* input) {
  // the reference builds its two FFTW plans here (src/FFT1D.cpp:14-54); the
  // device pass needs no plan, only the size and stride
  m_N = N;
  m_stride = stride;
  m_alignment = (int)((uintptr_t)input % 16);
}

void FFT1D::forward(cdouble* input, int N, int stride) { run_line(input, N, stride, -1, 1.0); }

void FFT1D::inverse(cdouble* input, int N, int stride) {
  // transform(+1) then divide by N (src/FFT1D.cpp:60-67); 1/N is exact for the
  // power-of-two lengths the device pass supports
  run_line(input, N, stride, +1, 1.0 / N);
}

void FFT1D::transform(cdouble* input, int N, int stride, int DIR) {
  run_line(input, N, stride, DIR == 1 ? 1 : -1, 1.0);
}

void FFT1D::transform(cdouble* input, int DIR) {
  run_line(input, m_N, m_stride, DIR == 1 ? 1 : -1, 1.0);
}
