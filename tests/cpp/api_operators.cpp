// Known-answer checks of the reference's test/operators.cpp (checks at
// test/operators.cpp:31-198, 1e-3 absolute) written against the same field
// API, with a non-zero exit status on failure.  Built against
// libspectral_b200.so by tests/test_gpu_api.py.
#include <cmath>
#include <iostream>

#include "DataObjects.H"

static int failures = 0;
static void report(const char* what, bool wrong) {
  std::cout << what << (wrong ? " failed" : " passed") << std::endl;
  if (wrong) failures++;
}

int main(int argc, char* argv[]) {
  upcxx::init();
  INT N = argc > 1 ? atoi(argv[1]) : 32;
  array<INT, DIM> dims = {N, N, N};
  Scalar s(dims);
  array<INT, DIM> ind = {0, 0, 0};
  for (ind[2] = 0; ind[2] < N; ind[2]++)
    for (ind[1] = 0; ind[1] < N; ind[1]++)
      for (ind[0] = 0; ind[0] < N; ind[0]++) s[ind] = sin(2 * M_PI / N * ind[0]);
  Scalar s_f(dims);
  s.forward(s_f);
  auto all = [&](auto pred) {
    bool wrong = false;
    for (ind[2] = 0; ind[2] < N; ind[2]++)
      for (ind[1] = 0; ind[1] < N; ind[1]++)
        for (ind[0] = 0; ind[0] < N; ind[0]++)
          if (pred()) wrong = true;
    return wrong;
  };
  const Scalar& cs = s;
  Scalar sum = s + s;
  report("addition", all([&] { return std::abs(sum[ind].real() - 2 * sin(2 * M_PI / N * ind[0])) > 1e-3; }));
  Scalar sub = s - s;
  report("subtraction", all([&] { return std::abs(sub[ind].real()) > 1e-3; }));
  Vector grad = s_f.gradient();
  grad.inverse();
  report("gradient", all([&] {
           return std::abs(grad[0][ind].real() - cos(2 * M_PI / N * ind[0])) > 1e-3 ||
                  std::abs(grad[1][ind].real()) > 1e-3 || std::abs(grad[2][ind].real()) > 1e-3;
         }));
  Scalar lap = s_f.laplacian();
  lap.inverse();
  report("laplacian", all([&] { return std::abs(lap[ind].real() + sin(2 * M_PI / N * ind[0])) > 1e-3; }));
  Scalar lap_inv;
  lap.forward(lap_inv);
  lap_inv.laplacian_inverse();
  lap_inv.inverse();
  report("laplacian inverse", all([&] { return std::abs(lap_inv[ind].real() - cs[ind].real()) > 1e-3; }));
  Vector v(dims);
  v[0] = s;
  v.forward();
  Scalar div = v.divergence();
  div.inverse();
  report("divergence", all([&] { return std::abs(div[ind].real() - cos(2 * M_PI / N * ind[0])) > 1e-3; }));
  Vector vlap = v.laplacian();
  vlap.inverse();
  report("vector laplacian", all([&] { return std::abs(vlap[0][ind].real() + sin(2 * M_PI / N * ind[0])) > 1e-3; }));
  Vector v1(dims), v2(dims);
  for (INT i = 0; i < v1[0].localSize(); i++) {
    v1[2][i] = 1.;
    v2[1][i] = 1.;
  }
  v1.forward();
  v2.forward();
  Vector cr = v1.cross(v2);
  cr.inverse();
  report("cross", all([&] {
           return std::abs(cr[0][ind].real() + 1) > 1e-3 || std::abs(cr[1][ind].real()) > 1e-3 ||
                  std::abs(cr[2][ind].real()) > 1e-3;
         }));
  grad.forward();
  Vector curl = grad.curl();
  curl.inverse();
  bool wrong = false;
  for (int d = 0; d < DIM; d++)
    for (INT i = 0; i < curl[0].localSize(); i++)
      if (std::abs(curl[d][i].real()) > 1e-3) wrong = true;
  report("curl", wrong);
  curl.forward();
  Vector mult = 2. * curl;
  report("double * vector", all([&] {
           for (int d = 0; d < DIM; d++)
             if (std::abs(mult[d][ind] - 2. * curl[d][ind]) > 1e-3) return true;
           return false;
         }));
  // Vector::isPhysical() is always false in the reference; arithmetic results are Fourier
  Vector p(dims);
  report("isPhysical quirk", p.isPhysical() || !(p + p).isFourier());
  upcxx::finalize();
  return failures ? 1 : 0;
}
