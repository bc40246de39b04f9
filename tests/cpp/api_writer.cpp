// Writer through the reference API: a physical scalar, a Fourier-space copy of
// it and a physical vector, written every second call of write() for five
// calls; the scalar grows by 1 after every call, so file w holds f + 2 w.
// Usage: api_writer <path prefix>
#include <cmath>

#include "DataObjects.H"
#include "Writer.H"

int main(int argc, char* argv[]) {
  upcxx::init();
  const string prefix = argc > 1 ? argv[1] : "writer_test";
  array<INT, DIM> dims = {8, 4, 16};
  Scalar s(dims);
  Vector v(dims);
  for (INT k = 0; k < dims[2]; k++)
    for (INT j = 0; j < dims[1]; j++)
      for (INT i = 0; i < dims[0]; i++) {
        const INT n = i + dims[0] * (j + dims[1] * k);
        s[n] = cdouble(std::sin(0.7 * i) + 0.1 * j - 0.3 * k, 0.0);
        v[0][n] = cdouble(i, 0.0);
        v[1][n] = cdouble(10 * j, 0.0);
        v[2][n] = cdouble(100 * k, 0.0);
      }
  Scalar g = s;
  g.forward();
  Writer writer(prefix);
  writer.add(s, "s");
  writer.add(g, "g");
  writer.add(v, "velocity");
  writer.setFreq(2);
  for (int t = 0; t < 5; t++) {
    writer.write();
    for (INT n = 0; n < s.localSize(); n++) s[n] += 1.0;
  }
  upcxx::finalize();
  return 0;
}
