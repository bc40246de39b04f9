// The exec/ns.cpp call sequence (bootstrap ns.cpp:132-153, loop
// ns.cpp:167-217) driven through the field API from a Taylor-Green or
// vortex-tube start; writes V1, omega1 and cross0 (interleaved complex
// doubles, x fastest) after `steps` steps to a binary file for comparison.
// Usage: api_ns_dump N steps nu K tg|vx out.bin
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>

#include "DataObjects.H"

int main(int argc, char* argv[]) {
  if (argc < 7) return 2;
  upcxx::init();
  INT N = atoi(argv[1]);
  int steps = atoi(argv[2]);
  double nu = atof(argv[3]), K = atof(argv[4]);
  bool tg = std::strcmp(argv[5], "tg") == 0;
  array<INT, DIM> dims = {N, N, N};
  Vector omega0(dims, !tg), omega1(dims, false), omega(dims, false);
  Vector V0(dims, false), V1(dims, false), V(dims, false), Vhalf(dims, false);
  Scalar Pi0(dims, false), Pi1(dims, false), G(dims, false), div(dims, false);
  array<INT, DIM> ind;
  const double h = 2 * M_PI / N;
  if (tg) {
    Vector u(dims);
    for (ind[2] = 0; ind[2] < N; ind[2]++)
      for (ind[1] = 0; ind[1] < N; ind[1]++)
        for (ind[0] = 0; ind[0] < N; ind[0]++) {
          double x = h * ind[0], y = h * ind[1], z = h * ind[2];
          u[0][ind] = sin(x) * cos(y) * cos(z);
          u[1][ind] = -cos(x) * sin(y) * cos(z);
        }
    u.forward();
    V0 = u;
    omega0 = V0.curl();
  } else {
    const double width = M_PI / 8, mag = 50, dist = M_PI / 2;
    auto gs = [&](double x, double y, double xc, double yc) {
      return exp(-pow(x - xc, 2) / width) * exp(-pow(y - yc, 2) / width);
    };
    for (ind[2] = 0; ind[2] < N; ind[2]++)
      for (ind[1] = 0; ind[1] < N; ind[1]++)
        for (ind[0] = 0; ind[0] < N; ind[0]++) {
          double x = h * ind[0], y = h * ind[1];
          omega0[2][ind] = mag * gs(x, y, M_PI - dist, M_PI - dist) +
                           mag * gs(x, y, M_PI + dist, M_PI - dist) + mag * gs(x, y, M_PI, M_PI + dist);
        }
    omega0.forward();
    Scalar psi(dims, false);
    for (ind[2] = 0; ind[2] < N; ind[2]++)
      for (ind[1] = 0; ind[1] < N; ind[1]++)
        for (ind[0] = 0; ind[0] < N; ind[0]++) {
          array<double, DIM> k = psi.freq(ind);
          if (k[0] != 0 || k[1] != 0) psi[ind] = -1. / (k[0] * k[0] + k[1] * k[1]) * omega0[2][ind];
        }
    Vector grad = psi.gradient();
    V0[0] = -1. * grad[1];
    V0[1] = grad[0];
  }
  Pi0 = (V0.cross(omega0) + nu * V0.laplacian()).divergence();
  Pi0.laplacian_inverse();
  V1 = V0 + K * (V0.cross(omega0) + nu * V0.laplacian() - Pi0.gradient());
  omega1 = V1.curl();
  Vector F;
  Vector cross0 = V0.cross(omega0);
  Vector cross1, lap1;
  for (int t = 1; t < steps + 1; t++) {
    cross1 = V1.cross(omega1);
    F = K / 2 * (3. * cross1 - cross0);
    lap1 = nu * K / 2 * V1.laplacian();
    G = (V1 + lap1 + F).divergence();
    G.laplacian_inverse();
    Vhalf = V1 + F - G.gradient();
    V = Vhalf + lap1;
    for (int d = 0; d < DIM; d++) V[d].laplacian_inverse(1, -nu * K / 2);
    omega = V.curl();
    div = V.divergence();
    if (div.average() > 1e-12) cout << "avg div = " << div.average() << endl;
    V0 = V1;
    V1 = V;
    omega0 = omega1;
    omega1 = omega;
    cross0 = cross1;
  }
  std::ofstream out(argv[6], std::ios::binary);
  for (const Vector* vec : {&V1, &omega1, &cross0})
    for (int d = 0; d < DIM; d++)
      for (INT i = 0; i < (*vec)[d].localSize(); i++) {
        cdouble c = (*vec)[d][i];
        out.write((const char*)&c, sizeof(c));
      }
  upcxx::finalize();
  return 0;
}
