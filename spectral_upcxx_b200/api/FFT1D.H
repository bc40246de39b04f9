#ifndef __FFT_1D_H__
#define __FFT_1D_H__

// B200 replacement of the reference's FFT1D (src/FFT1D.H:18-47).  Same
// public signatures; the transform runs on the GPU through sns_fft1d_many
// (include/spectral_b200.h).  A pointer to device memory is transformed in
// place on the device; a host pointer is staged through a device buffer, so
// code that hands FFT1D host lines keeps working.

#include <array>
#include <complex>
#include <cstdint>
#include <vector>

#ifndef DIM
#define DIM 3
#endif

using namespace std;

typedef complex<double> cdouble;
typedef uint64_t INT;

/// do FFT in 1 dimension
class FFT1D {
 public:
  /// default constructor
  FFT1D();
  /// set stride and size to reuse plan (the pointer only fixes the layout)
  void init(int N, int stride, cdouble* input);
  /// destructor
  ~FFT1D();
  /// in place forward transform on data of size N with stride stride
  void forward(cdouble* input, int N, int stride = 1);
  /// in place inverse transform on data of size N with stride stride (divides by N)
  void inverse(cdouble* input, int N, int stride = 1);
  /// in place transform: dir = -1 is exp(-i..), dir = +1 is exp(+i..), unnormalised
  void transform(cdouble* input, int N, int stride, int dir);
  /// in place transform with the size and stride given to init
  void transform(cdouble* input, int DIR);

 private:
  int m_N;
  int m_stride;
  int m_dir;
  int m_alignment;
};

#endif
