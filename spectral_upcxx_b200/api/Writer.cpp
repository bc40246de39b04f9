// Output registry with the reference's interface (src/Writer.cpp:6-169).
// VTK file output is outside the GPU hot path; write() only counts the calls
// that the reference would turn into files.
#include "Writer.H"

Writer::Writer(string name) : m_name(name), m_count(0), m_writes(0), m_f(1) {}

Writer::~Writer() {}

void Writer::add(Scalar& a_scalar, string a_name) {
  m_scalars.push_back(&a_scalar);
  m_scalar_names.push_back(a_name);
}

void Writer::add(Vector& a_vector, string a_name) {
  m_vectors.push_back(&a_vector);
  m_vector_names.push_back(a_name);
}

void Writer::setFreq(int a_f) { m_f = a_f; }

void Writer::write() {
  // the reference computes m_count++ % m_f (src/Writer.cpp:39), which faults
  // for the m_f = 0 that exec/ns.cpp sets; a frequency <= 0 writes nothing
  if (m_f <= 0) {
    m_count++;
    return;
  }
  if (m_count++ % m_f != 0) return;
  m_writes++;
}
