#ifndef _OPERATORS_H_
#define _OPERATORS_H_

// Element-wise operators of the reference (src/Operators.H:4-17), each a
// device kernel returning a new field.

Scalar operator*(const Scalar& a, const Scalar& b);
Scalar operator-(const Scalar& a, const Scalar& b);
Scalar operator+(const Scalar& a, const Scalar& b);
Vector operator-(const Vector& a, const Vector& b);
Vector operator+(const Vector& a, const Vector& b);
Scalar operator*(double alpha, const Scalar& s);
Vector operator*(double alpha, const Vector& v);

#endif
