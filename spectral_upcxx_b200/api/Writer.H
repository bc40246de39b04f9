#ifndef _WRITER_H_
#define _WRITER_H_

// Output registry with the reference's interface (src/Writer.H:12-48): every
// m_f-th write() stores the registered fields, in physical space, as one
// legacy-VTK rectilinear-grid file "<name>0_<w>.vtk" (ASCII, point data,
// scalars then vectors, as src/Writer.cpp:35-168 lays them out through its
// VisIt writer) and lists it in "<name>.visit" (!NBLOCKS 1).  The device
// fields are inverse-transformed and copied to the host during write(); the
// text formatting and the file writing run on a background thread, so the
// time loop continues meanwhile (one file in flight; the next write() and the
// destructor wait for it).  A write frequency of 0 -- which exec/ns.cpp:47-52
// sets and which makes the reference divide by zero (src/Writer.cpp:39) --
// writes nothing.  The master file is created at the first file, not in the
// constructor, so a writer that never writes leaves no file behind.  With
// NWRITE defined nothing is written, as in the reference.

#include <fstream>
#include <string>
#include <thread>
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
  void wait_pending();

  string m_name;
  int m_count;
  int m_writes;
  vector<Scalar*> m_scalars;
  vector<string> m_scalar_names;
  vector<Vector*> m_vectors;
  vector<string> m_vector_names;
  int m_f;
  ofstream m_out;
  thread m_job;
};

#endif
