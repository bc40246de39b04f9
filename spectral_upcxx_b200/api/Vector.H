#ifndef _VECTOR_H_
#define _VECTOR_H_

// B200 replacement of the reference's Vector (src/Vector.H:5-70): three
// Scalars.  Same public interface; operators run as device kernels.

/// Represent a vector with scalars in DIM directions
class Vector {
 public:
  Vector();
  /// supply Nx, Ny, Nz. Defaults to building in physical space
  Vector(array<INT, DIM> dims, bool physical = true);
  void init(array<INT, DIM> dims, bool physical = true);
  Scalar& operator[](int a_i);
  const Scalar& operator[](int a_i) const;

  void forward();
  void inverse();
  void forward(Vector& a_vector) const;
  void inverse(Vector& a_vector) const;

  /// (*this) x a_v, formed in physical space, returned in fourier space
  Vector cross(const Vector& a_v) const;
  /// curl, fourier space in and out
  Vector curl() const;
  /// divergence, fourier space in and out
  Scalar divergence() const;
  /// vector laplacian, fourier space in and out
  Vector laplacian() const;

  bool isFourier() const;
  /// always false, as in the reference (src/Vector.cpp:191-197)
  bool isPhysical() const;

  INT localSize() const;
  array<INT, DIM> getDims() const;
  array<INT, DIM> getPStart() const;
  array<INT, DIM> getPEnd() const;
  array<INT, DIM> getPDims() const;

 private:
  void setFourier();
  void setPhysical();
  array<INT, DIM> m_dims;
  INT m_N;
  array<Scalar, DIM> m_vector;
};

#endif
