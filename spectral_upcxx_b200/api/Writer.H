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
//
// Final state: with the environment variable SNS_WRITER_FINAL set to a path
// prefix, every live writer also writes its registered fields once more, at
// upcxx::finalize() (when a driver's fields still exist), to
// "<prefix><name>.vtk" in the same format -- whatever the write frequency, so
// a run made with frequency 0 still leaves its last state behind.

#include <fstream>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "DataObjects.H"

using namespace std;

// one registered field copied to the host (defined with the writer)
struct SnsWriterField;

class Writer {
 public:
  Writer(string name = "solution");
  ~Writer();
  void add(Scalar& a_scalar, string a_name);
  void add(Vector& a_vector, string a_name);
  void write();
  void setFreq(int a_f);
  /// write the registered fields now, synchronously, to the file `fname`
  void writeFile(const string& fname);
  const string& name() const { return m_name; }
  /// number of registered scalars and vectors
  size_t fields() const { return m_scalars.size() + m_vectors.size(); }

 private:
  void wait_pending();
  std::shared_ptr<vector<SnsWriterField>> collect(array<INT, DIM>& dims,
                                                    array<INT, DIM>& pdims) const;

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
