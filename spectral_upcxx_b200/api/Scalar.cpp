// Scalar on the GPU: the reference's src/Scalar.cpp semantics over the
// spectral_b200 C-ABI.  Device work is queued on the legacy default stream,
// so host mirror copies (synchronous cudaMemcpy) order after it.
#include <cuda_runtime.h>

#include <cstring>
#include <iostream>
#include <vector>

#include "DataObjects.H"
#include "sns_api_internal.H"

namespace {
int g_prec = -1;
int g_zero = -1;

size_t elem_bytes(int prec) { return prec == SNS_C128 ? 16 : 8; }
}  // namespace

namespace sns_api {
int precision() {
  if (g_prec < 0) {
    const char* e = std::getenv("SNS_PRECISION");
    g_prec = (e && (std::strcmp(e, "fp32") == 0 || std::strcmp(e, "c64") == 0)) ? SNS_C64
                                                                                  : SNS_C128;
  }
  return g_prec;
}
void set_precision(int prec) { g_prec = (prec == SNS_C64) ? SNS_C64 : SNS_C128; }
bool zero_high_modes() {
  if (g_zero < 0) {
    const char* e = std::getenv("SNS_ZERO");
    g_zero = (e && std::strcmp(e, "0") == 0) ? 0 : 1;
  }
  return g_zero == 1;
}
void set_zero_high_modes(bool on) { g_zero = on ? 1 : 0; }
void synchronize() { SNS_API_CHECK(sns_stream_synchronize(nullptr)); }
}  // namespace sns_api

int Scalar::m_nscalars = 0;

Scalar::Scalar()
    : m_dims{0, 0, 0},
      m_pdims{0, 0, 0},
      m_N(0),
      m_dSize(0),
      m_prec(SNS_C128),
      m_dev(nullptr),
      m_host(nullptr),
      m_sync(0),
      m_fourier(false),
      m_initialized(false) {}

Scalar::Scalar(array<INT, DIM> N, bool physical) : Scalar() { init(N, physical); }

Scalar::~Scalar() { release(); }

void Scalar::release() {
  if (m_initialized) {
    sns_free(m_dev);
    delete[] m_host;
    m_dev = nullptr;
    m_host = nullptr;
    m_nscalars--;
    m_initialized = false;
  }
}

Scalar::Scalar(const Scalar& scalar) : Scalar() {
  if (!scalar.m_initialized) return;
  init(scalar.getDims(), scalar.isPhysical());
  *this = scalar;
}

void Scalar::operator=(const Scalar& scalar) {
  if (this == &scalar || !scalar.m_initialized) return;
  if (!m_initialized) init(scalar.getDims(), scalar.isPhysical());
  if (scalar.m_N != m_N) SNS_API_ERROR("assignment between fields of different sizes");
  if (scalar.m_sync == 1 && m_prec == scalar.m_prec) {
    // the source's host copy is the current one: copy it and upload lazily
    if (!m_host) m_host = new cdouble[m_dSize];
    std::memcpy((void*)m_host, (const void*)scalar.m_host, m_dSize * sizeof(cdouble));
    m_sync = 1;
    return;
  }
  const void* src = scalar.devRead();
  SNS_API_CHECK(sns_convert(m_dev, m_prec, src, scalar.m_prec, (int64_t)m_N, nullptr));
  m_sync = 0;
}

void Scalar::init(array<INT, DIM> N, bool physical) {
  release();
  m_initialized = true;
  m_nscalars++;
  m_dims = N;
  m_N = 1;
  for (int i = 0; i < DIM; i++) m_N *= m_dims[i];
  m_pdims = {m_dims[0], m_dims[1], m_dims[2]};
  m_dSize = m_N;
  m_prec = sns_api::precision();
  SNS_API_CHECK(sns_malloc(&m_dev, elem_bytes(m_prec) * m_N));
  // the reference value-initialises its storage (upcxx::new_array)
  SNS_API_CHECK(sns_memset(m_dev, 0, elem_bytes(m_prec) * m_N, nullptr));
  m_sync = 0;
  if (physical)
    setPhysical();
  else
    setFourier();
}

void Scalar::ensure_host() const {
  if (!m_host) {
    m_host = new cdouble[m_dSize];
    if (m_sync == 1) m_sync = 0;  // nothing was written to a mirror that did not exist
  }
  if (m_sync != 0) return;
  if (m_prec == SNS_C128) {
    SNS_API_CHECK(sns_memcpy_d2h(m_host, m_dev, m_N * sizeof(cdouble), nullptr));
  } else {
    std::vector<float> buf(2 * m_N);
    SNS_API_CHECK(sns_memcpy_d2h(buf.data(), m_dev, buf.size() * sizeof(float), nullptr));
    for (INT i = 0; i < m_N; i++) m_host[i] = cdouble(buf[2 * i], buf[2 * i + 1]);
  }
  SNS_API_CHECK(sns_stream_synchronize(nullptr));
  m_sync = 2;
}

void Scalar::ensure_device() const {
  if (m_sync != 1) return;
  if (m_prec == SNS_C128) {
    SNS_API_CHECK(sns_memcpy_h2d(m_dev, m_host, m_N * sizeof(cdouble), nullptr));
    SNS_API_CHECK(sns_stream_synchronize(nullptr));
  } else {
    std::vector<float> buf(2 * m_N);
    for (INT i = 0; i < m_N; i++) {
      buf[2 * i] = (float)m_host[i].real();
      buf[2 * i + 1] = (float)m_host[i].imag();
    }
    SNS_API_CHECK(sns_memcpy_h2d(m_dev, buf.data(), buf.size() * sizeof(float), nullptr));
    SNS_API_CHECK(sns_stream_synchronize(nullptr));
  }
  m_sync = 2;
}

const void* Scalar::devRead() const {
  if (!m_initialized) SNS_API_ERROR("field used before init");
  ensure_device();
  return m_dev;
}
void* Scalar::devWrite() {
  if (!m_initialized) SNS_API_ERROR("field used before init");
  m_sync = 0;
  return m_dev;
}
void* Scalar::devReadWrite() {
  if (!m_initialized) SNS_API_ERROR("field used before init");
  ensure_device();
  m_sync = 0;
  return m_dev;
}

INT Scalar::index_of(array<INT, DIM> index) const {
  INT n = index[0] + m_dims[0] * index[1] + index[2] * m_dims[0] * m_dims[1];
  if (n >= m_N) {
    cout << n << endl;
    SNS_API_ERROR("indexing out of full dimensions");
  }
  return n;
}

void Scalar::set(array<INT, DIM> index, cdouble val) {
  INT loc = index_of(index);
  ensure_host();
  m_host[loc] = val;
  m_sync = 1;
}

cdouble Scalar::get(array<INT, DIM> index) const {
  INT loc = index_of(index);
  ensure_host();
  return m_host[loc];
}

cdouble& Scalar::operator[](array<INT, DIM> index) {
  INT loc = index_of(index);
  ensure_host();
  m_sync = 1;
  return m_host[loc];
}

cdouble Scalar::operator[](array<INT, DIM> index) const {
  INT loc = index_of(index);
  ensure_host();
  return m_host[loc];
}

cdouble& Scalar::operator()(INT a_i, INT a_j, INT a_k) {
  array<INT, DIM> index = {a_i, a_j, a_k};
  return (*this)[index];
}

cdouble Scalar::operator()(INT a_i, INT a_j, INT a_k) const {
  array<INT, DIM> index = {a_i, a_j, a_k};
  return (*this)[index];
}

cdouble& Scalar::operator[](INT index) {
  if (index >= m_dSize) SNS_API_ERROR("accessed out of local data");
  ensure_host();
  m_sync = 1;
  return m_host[index];
}

cdouble Scalar::operator[](INT index) const {
  if (index >= m_dSize) SNS_API_ERROR("accessed out of local data");
  ensure_host();
  return m_host[index];
}

array<double, DIM> Scalar::freq(array<INT, DIM> ind) const {
  array<double, DIM> k;
  for (int i = 0; i < DIM; i++) {
    if (ind[i] <= m_dims[i] / 2)
      k[i] = (double)ind[i];
    else
      k[i] = -1. * (double)m_dims[i] + (double)ind[i];
  }
  return k;
}

void Scalar::forward() {
  if (isFourier()) SNS_API_ERROR("already in fourier space");
  const int flags = sns_api::zero_high_modes() ? SNS_FFT_ZERO_NYQUIST : 0;
  SNS_API_CHECK(sns_fft3d(devReadWrite(), m_dims[0], m_dims[1], m_dims[2], -1, flags, m_prec,
                          nullptr));
  setFourier();
}

void Scalar::inverse() {
  if (isPhysical()) SNS_API_ERROR("already in physical space");
  SNS_API_CHECK(sns_fft3d(devReadWrite(), m_dims[0], m_dims[1], m_dims[2], +1,
                          SNS_FFT_NORMALISE, m_prec, nullptr));
  setPhysical();
}

void Scalar::forward(Scalar& a_scalar) const {
  a_scalar = (*this);
  a_scalar.forward();
}

void Scalar::inverse(Scalar& a_scalar) const {
  a_scalar = (*this);
  a_scalar.inverse();
}

Vector Scalar::gradient() const {
  if (!isFourier()) SNS_API_ERROR("must begin gradient in fourier space");
  Vector v(m_dims, false);
  SNS_API_CHECK(sns_gradient(devRead(), v[0].devWrite(), v[1].devWrite(), v[2].devWrite(),
                             m_dims[0], m_dims[1], m_dims[2], m_prec, nullptr));
  return v;
}

Scalar Scalar::laplacian() const {
  if (!isFourier()) SNS_API_ERROR("must begin laplacian in fourier space");
  Scalar lap(m_dims, false);
  SNS_API_CHECK(
      sns_laplacian(devRead(), lap.devWrite(), m_dims[0], m_dims[1], m_dims[2], m_prec, nullptr));
  return lap;
}

void Scalar::laplacian_inverse(double a, double b) {
  SNS_API_CHECK(sns_laplacian_inverse(devReadWrite(), a, b, m_dims[0], m_dims[1], m_dims[2],
                                      m_prec, nullptr));
}

void Scalar::zeroHighModes() {
  if (!sns_api::zero_high_modes()) return;
  SNS_API_CHECK(
      sns_zero_high_modes(devReadWrite(), m_dims[0], m_dims[1], m_dims[2], m_prec, nullptr));
}

INT Scalar::localSize() const { return m_dSize; }
array<INT, DIM> Scalar::getDims() const { return m_dims; }
array<INT, DIM> Scalar::getPDims() const { return m_pdims; }
array<INT, DIM> Scalar::getPStart() const {
  array<INT, DIM> start = {0, 0, 0};
  return start;
}
array<INT, DIM> Scalar::getPEnd() const {
  array<INT, DIM> end = {m_dims[0], m_dims[1], m_dims[2]};
  return end;
}
INT Scalar::size() const { return m_N; }
double Scalar::memory() const {
  double mem = (double)m_nscalars * (double)m_N * elem_bytes(m_prec) / 1e9;
  cout << "memory requirement = " << mem << " GB" << endl;
  return mem;
}

void Scalar::setPhysical() { m_fourier = false; }
void Scalar::setFourier() { m_fourier = true; }
bool Scalar::isPhysical() const { return !m_fourier; }
bool Scalar::isFourier() const { return m_fourier; }

double Scalar::average() const {
  double avg = 0;
  SNS_API_CHECK(sns_average_abs(devRead(), (int64_t)m_N, m_prec, &avg, nullptr));
  return avg;
}
