#ifndef _PARTICLE_H_
#define _PARTICLE_H_

// Tracer particle with the reference's interface (src/Particle.H:5-17);
// exec/ns.cpp includes it and uses it only when built with PARTICLES.

#include "DataObjects.H"

class Particle {
 public:
  Particle();
  void move(const Vector& velocity, double K);
  double energy();
  array<double, DIM> position();

 private:
  array<double, DIM> m_loc;
  array<double, DIM> m_v;
};

#endif
