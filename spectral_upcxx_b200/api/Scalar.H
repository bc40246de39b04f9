#ifndef __SCALAR_H__
#define __SCALAR_H__

// B200 replacement of the reference's Scalar (src/Scalar.H:10-145): a 3D
// complex field resident in HBM.  The public interface is the reference's,
// signature for signature, so exec/ns.cpp and test/operators.cpp compile
// against it unchanged.  Storage is a device buffer from the library's
// caching pool (complex128, or complex64 when SNS_PRECISION=fp32) plus a lazily
// synchronised complex<double> host mirror behind element access.  One process
// owns the whole box (the reference's z-slab decomposition collapses to one
// slab), so every index is local.

#include "FFT1D.H"

class Vector;

/// Store a 3D array on the GPU
class Scalar {
 public:
  /// default constructor
  Scalar();
  /// constructor: set size in DIM directions. Defaults to building in physical space
  Scalar(array<INT, DIM> N, bool physical = true);
  /// destructor
  ~Scalar();
  /// copy constructor (deep copy)
  Scalar(const Scalar& scalar);
  /// copy assignment. Does a deep copy; an initialised target keeps its flag
  void operator=(const Scalar& scalar);
  /// initialize the array after calling default constructor
  void init(array<INT, DIM> N, bool physical = true);
  /// set a value in the array
  void set(array<INT, DIM> index, cdouble val);
  /// get a value from the array
  cdouble get(array<INT, DIM> index) const;
  /// element access (host mirror)
  cdouble& operator[](array<INT, DIM> index);
  cdouble operator[](array<INT, DIM> index) const;
  cdouble& operator()(INT a_i, INT a_j, INT a_k);
  cdouble operator()(INT a_i, INT a_j, INT a_k) const;
  cdouble& operator[](INT index);
  cdouble operator[](INT index) const;
  /// return frequency for grid point ind
  array<double, DIM> freq(array<INT, DIM> ind) const;

  /// in place forward transform (then zeroHighModes)
  void forward();
  /// in place reverse transform (divides by N)
  void inverse();
  /// out of place forward transform
  void forward(Scalar& a_scalar) const;
  /// out of place reverse transform
  void inverse(Scalar& a_scalar) const;

  /// gradient, returned in fourier space
  Vector gradient() const;
  /// laplacian, returned in fourier space
  Scalar laplacian() const;
  /// invert a + b*laplacian: divides by a - b(m^2 + n^2 + p^2) where that sum != 0
  void laplacian_inverse(double a = 0, double b = 1);
  /// zero out the highest modes
  void zeroHighModes();

  INT localSize() const;
  array<INT, DIM> getDims() const;
  array<INT, DIM> getPDims() const;
  array<INT, DIM> getPStart() const;
  array<INT, DIM> getPEnd() const;
  INT size() const;
  double memory() const;

  bool isPhysical() const;
  bool isFourier() const;
  void setFourier();
  void setPhysical();

  /// mean of |f_i|
  double average() const;

  // ---- device access (no counterpart in the reference) ----
  /// device data, valid for reading (uploads host edits first)
  const void* devRead() const;
  /// device data that the caller overwrites completely (host mirror dropped)
  void* devWrite();
  /// device data read and modified in place
  void* devReadWrite();
  /// storage precision (SNS_C64 or SNS_C128)
  int precision() const { return m_prec; }

 private:
  void ensure_host() const;
  void ensure_device() const;
  void release();
  INT index_of(array<INT, DIM> index) const;

  array<INT, DIM> m_dims;
  array<INT, DIM> m_pdims;
  INT m_N;
  INT m_dSize;
  int m_prec;
  void* m_dev;
  mutable cdouble* m_host;
  // 0: device copy current, host stale; 1: host edited, device stale; 2: both current
  mutable int m_sync;
  bool m_fourier;
  bool m_initialized;
  static int m_nscalars;
};

#endif
