// exec/ns.cpp's particle loop (ns.cpp:157-203, PARTICLES) through the
// Particle class of the API: srand(seed), np particles at random positions,
// nsteps moves through a physical velocity field held in a device Vector.
// The velocity (3 complex-double fields, x fastest) is read from `vel.bin`;
// initial positions, final positions and energies are written to `out.bin`
// as doubles.
// Usage: api_particles seed np nx ny nz K nsteps vel.bin out.bin
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "DataObjects.H"
#include "Particle.H"

int main(int argc, char* argv[]) {
  if (argc < 10) return 2;
  upcxx::init();
  const unsigned seed = (unsigned)atoi(argv[1]);
  const long np = atol(argv[2]);
  const INT nx = atoi(argv[3]), ny = atoi(argv[4]), nz = atoi(argv[5]);
  const double K = atof(argv[6]);
  const int nsteps = atoi(argv[7]);
  array<INT, DIM> dims = {nx, ny, nz};
  Vector vel(dims);
  {
    FILE* f = fopen(argv[8], "rb");
    if (!f) return 3;
    std::vector<cdouble> buf(nx * ny * nz);
    for (int d = 0; d < DIM; d++) {
      if (fread(buf.data(), sizeof(cdouble), buf.size(), f) != buf.size()) return 4;
      for (INT i = 0; i < buf.size(); i++) vel[d][i] = buf[i];
    }
    fclose(f);
  }
  srand(seed);
  std::vector<Particle> parts(np);
  std::vector<double> out;
  for (long p = 0; p < np; p++)
    for (double x : parts[p].position()) out.push_back(x);
  for (int t = 0; t < nsteps; t++)
    for (long p = 0; p < np; p++) parts[p].move(vel, K);
  for (long p = 0; p < np; p++)
    for (double x : parts[p].position()) out.push_back(x);
  for (long p = 0; p < np; p++) out.push_back(parts[p].energy());
  FILE* f = fopen(argv[9], "wb");
  if (!f) return 5;
  fwrite(out.data(), sizeof(double), out.size(), f);
  fclose(f);
  upcxx::finalize();
  return 0;
}
