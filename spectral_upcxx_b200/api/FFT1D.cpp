// FFT1D over the device line-FFT pass (sns_fft1d_many).  The reference runs
// one FFTW plan per strided line (src/FFT1D.cpp:14-101); here a device line
// is transformed on the device in place, and a host line is staged through a
// device buffer.
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

// Transform one line of N elements `stride` apart in place, then multiply by
// `scale` (1 for the unnormalised transforms, 1/N for inverse()).
void run_line(cdouble* input, int N, int stride, int dir, double scale) {
  if (N < 1 || stride < 1) {
    std::cerr << "ERROR in FFT1D: bad size or stride" << std::endl;
    std::exit(1);
  }
  const size_t bytes = sizeof(cdouble) * (size_t)N;
  void* d = nullptr;
  SNS_API_CHECK(sns_malloc(&d, bytes));
  const bool on_device = is_device_pointer(input);
  const cudaMemcpyKind in_kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind out_kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  // gather the (possibly strided) line into a contiguous device buffer
  if (cudaMemcpy2D(d, sizeof(cdouble), input, sizeof(cdouble) * (size_t)stride, sizeof(cdouble), N,
                   in_kind) != cudaSuccess) {
    std::cerr << "ERROR in FFT1D: line copy failed" << std::endl;
    std::exit(1);
  }
  SNS_API_CHECK(sns_fft1d_many(d, N, 1, 1, N, dir, SNS_C128, nullptr));
  if (scale != 1.0) SNS_API_CHECK(sns_axpby(scale, d, 0.0, nullptr, d, N, SNS_C128, nullptr));
  if (cudaMemcpy2D(input, sizeof(cdouble) * (size_t)stride, d, sizeof(cdouble), sizeof(cdouble), N,
                   out_kind) != cudaSuccess) {
    std::cerr << "ERROR in FFT1D: line copy failed" << std::endl;
    std::exit(1);
  }
  SNS_API_CHECK(sns_free(d));
}

}  // namespace

FFT1D::FFT1D() : m_N(0), m_stride(1), m_dir(0), m_alignment(0) {}
FFT1D::~FFT1D() {}

void FFT1D::init(int N, int stride, cdouble* input) {
  m_N = N;
  m_stride = stride;
  m_alignment = (int)((uintptr_t)input % 16);
}

void FFT1D::forward(cdouble* input, int N, int stride) { run_line(input, N, stride, -1, 1.0); }

void FFT1D::inverse(cdouble* input, int N, int stride) {
  // transform(+1) then divide by N (src/FFT1D.cpp:60-67)
  run_line(input, N, stride, +1, 1.0 / N);
}

void FFT1D::transform(cdouble* input, int N, int stride, int DIR) {
  run_line(input, N, stride, DIR == 1 ? 1 : -1, 1.0);
}

void FFT1D::transform(cdouble* input, int DIR) {
  run_line(input, m_N, m_stride, DIR == 1 ? 1 : -1, 1.0);
}
