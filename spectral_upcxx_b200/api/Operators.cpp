// Element-wise operators (src/Operators.cpp:9-99) as device kernels.  Each
// returns a new field from the caching pool, flagged as the reference flags
// it (Vector results take a.isPhysical(), which is always false).
#include "DataObjects.H"
#include "sns_api_internal.H"

namespace {
void axpby(double alpha, const Scalar& x, double beta, const Scalar* y, Scalar& out) {
  SNS_API_CHECK(sns_axpby(alpha, x.devRead(), beta, y ? y->devRead() : nullptr, out.devWrite(),
                          (int64_t)x.localSize(), x.precision(), nullptr));
}
}  // namespace

Scalar operator*(const Scalar& a, const Scalar& b) {
  if (a.isPhysical() != b.isPhysical()) SNS_API_ERROR("space mismatch");
  Scalar ret(a.getDims(), a.isPhysical());
  SNS_API_CHECK(sns_mul(a.devRead(), b.devRead(), ret.devWrite(), (int64_t)a.localSize(),
                        a.precision(), nullptr));
  return ret;
}

Scalar operator-(const Scalar& a, const Scalar& b) {
  if (a.isPhysical() != b.isPhysical()) SNS_API_ERROR("space mismatch");
  Scalar ret(a.getDims(), a.isPhysical());
  axpby(1.0, a, -1.0, &b, ret);
  return ret;
}

Scalar operator+(const Scalar& a, const Scalar& b) {
  if (a.isPhysical() != b.isPhysical()) SNS_API_ERROR("space mismatch");
  Scalar ret(a.getDims(), a.isPhysical());
  axpby(1.0, a, 1.0, &b, ret);
  return ret;
}

Vector operator-(const Vector& a, const Vector& b) {
  if (a.isPhysical() != b.isPhysical()) SNS_API_ERROR("space mismatch");
  Vector ret(a.getDims(), a.isPhysical());
  for (int d = 0; d < DIM; d++) axpby(1.0, a[d], -1.0, &b[d], ret[d]);
  return ret;
}

Vector operator+(const Vector& a, const Vector& b) {
  if (a.isPhysical() != b.isPhysical()) SNS_API_ERROR("space mismatch");
  Vector ret(a.getDims(), a.isPhysical());
  for (int d = 0; d < DIM; d++) axpby(1.0, a[d], 1.0, &b[d], ret[d]);
  return ret;
}

Scalar operator*(double alpha, const Scalar& s) {
  Scalar ret(s.getDims(), s.isPhysical());
  axpby(alpha, s, 0.0, nullptr, ret);
  return ret;
}

Vector operator*(double alpha, const Vector& v) {
  Vector ret(v.getDims(), v.isPhysical());
  for (int d = 0; d < DIM; d++) axpby(alpha, v[d], 0.0, nullptr, ret[d]);
  return ret;
}
