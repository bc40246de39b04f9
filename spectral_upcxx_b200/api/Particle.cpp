// Tracer particle (src/Particle.cpp:12-46 semantics): random start in
// [0, 2 pi]^3, trilinear interpolation of the physical velocity, periodic
// wrap.  Reads go through the host mirror of the velocity field.
#include "Particle.H"

#include <cmath>
#include <cstdlib>

Particle::Particle() {
  for (int i = 0; i < DIM; i++) m_loc[i] = (double)rand() / RAND_MAX * 2 * M_PI;
  m_v = {0, 0, 0};
}

void Particle::move(const Vector& velocity, double K) {
  array<INT, DIM> ind;
  array<INT, DIM> dims = velocity.getDims();
  array<double, DIM> h, rd;
  for (int d = 0; d < DIM; d++) {
    h[d] = 2 * M_PI / dims[d];
    ind[d] = (INT)(m_loc[d] / h[d]);
    if (ind[d] + 1 >= dims[d]) ind[d] = dims[d] - 2;
    rd[d] = (m_loc[d] - ind[d] * h[d]) / h[d];
  }
  // Corners in the order of the reference's sum (src/Particle.cpp:26-35): the
  // lower z face counter-clockwise from (0,0), then the upper z face; each term
  // is ((u * wx) * wy) * wz and the terms are added left to right, so the
  // rounding is the reference's.
  static const int corner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  for (int d = 0; d < DIM; d++) {
    const Scalar& u = velocity[d];
    double acc = 0;
    for (int c = 0; c < 8; c++) {
      const int ox = corner[c][0], oy = corner[c][1], oz = corner[c][2];
      const double t = u[array<INT, DIM>{ind[0] + ox, ind[1] + oy, ind[2] + oz}].real() *
                       (ox ? rd[0] : 1 - rd[0]) * (oy ? rd[1] : 1 - rd[1]) *
                       (oz ? rd[2] : 1 - rd[2]);
      acc = c == 0 ? t : acc + t;
    }
    m_v[d] = acc;
  }
  for (int d = 0; d < DIM; d++) {
    m_loc[d] += m_v[d] * K;
    if (m_loc[d] >= 2 * M_PI)
      m_loc[d] = m_loc[d] - 2 * M_PI;
    else if (m_loc[d] <= 0)
      m_loc[d] = 2 * M_PI + m_loc[d];
  }
}

double Particle::energy() {
  double e = 0;
  for (int d = 0; d < DIM; d++) e += m_v[d] * m_v[d];
  return .5 * e;
}

array<double, DIM> Particle::position() { return m_loc; }
