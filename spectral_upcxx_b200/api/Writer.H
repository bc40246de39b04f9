#ifndef _WRITER_H_
#define _WRITER_H_

// Output registry with the reference's interface (src/Writer.H:12-48).
// Field output (VTK files) is outside the GPU hot path: write() counts calls
// and returns, and a write frequency of 0 -- which exec/ns.cpp:47-52 sets and
// which makes the reference divide by zero (src/Writer.cpp:39) -- is safe.

#include <fstream>
#include <string>
#include <vector>

#include "DataObjects.H"

using namespace std;

class Writer {
 public:
  Writer(string name = "solution");
  ~Writer();
  void add(Scalar& a_scalar, string a_name);
  void add(Vector& a_vector, string a_name);
  void write();
  void setFreq(int a_f);

 private:
  string m_name;
  int m_count;
  int m_writes;
  vector<Scalar*> m_scalars;
  vector<string> m_scalar_names;
  vector<Vector*> m_vectors;
  vector<string> m_vector_names;
  int m_f;
};

#endif
