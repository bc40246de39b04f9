// Field output of the reference's Writer (src/Writer.cpp:6-169), written from
// the file-format description of legacy VTK (rectilinear grid, ASCII point
// data); see Writer.H for the behaviour.
#include "Writer.H"

#include <cmath>
#include <cstdio>
#include <memory>
#include <set>

#include "sns_api_internal.H"

// One field's physical values copied to the host: real parts only are kept
struct SnsWriterField {
  string name;
  int ncomp;               // 1 (scalar) or 3 (vector)
  vector<float> values;    // point-major: ncomp values per point, x fastest
};

namespace {

// Real parts of a device field (complex64 or complex128) into dst[i * stride]
void real_parts(const Scalar& s, float* dst, int stride) {
  const INT n = s.localSize();
  const int prec = s.precision();
  if (prec == SNS_C128) {
    vector<double> buf(2 * n);
    SNS_API_CHECK(sns_memcpy_d2h(buf.data(), s.devRead(), buf.size() * sizeof(double), nullptr));
    for (INT i = 0; i < n; i++) dst[i * stride] = (float)buf[2 * i];
  } else {
    vector<float> buf(2 * n);
    SNS_API_CHECK(sns_memcpy_d2h(buf.data(), s.devRead(), buf.size() * sizeof(float), nullptr));
    for (INT i = 0; i < n; i++) dst[i * stride] = buf[2 * i];
  }
}

void write_vtk(const string& fname, array<INT, DIM> dims, array<INT, DIM> pdims,
               const vector<SnsWriterField>& fields) {
  FILE* f = fopen(fname.c_str(), "w");
  if (!f) {
    std::cerr << "ERROR in Writer: cannot open " << fname << std::endl;
    return;
  }
  fprintf(f, "# vtk DataFile Version 2.0\nspectral_upcxx_b200 fields\nASCII\n");
  fprintf(f, "DATASET RECTILINEAR_GRID\nDIMENSIONS %d %d %d\n", (int)pdims[0], (int)pdims[1],
          (int)pdims[2]);
  // grid coordinates as src/Writer.cpp:129-141 sets them (y uses dims[0] too)
  const double b = 2 * M_PI;
  const char* axis[3] = {"X", "Y", "Z"};
  const INT den[3] = {dims[0], dims[0], dims[2]};
  for (int d = 0; d < 3; d++) {
    fprintf(f, "%s_COORDINATES %d float\n", axis[d], (int)pdims[d]);
    for (INT i = 0; i < pdims[d]; i++) fprintf(f, "%.9g\n", (float)(i * b / den[d]));
  }
  const INT npts = pdims[0] * pdims[1] * pdims[2];
  fprintf(f, "POINT_DATA %lld\n", (long long)npts);
  for (const SnsWriterField& h : fields) {
    if (h.ncomp == 1)
      fprintf(f, "SCALARS %s float\nLOOKUP_TABLE default\n", h.name.c_str());
    else
      fprintf(f, "VECTORS %s float\n", h.name.c_str());
    for (INT p = 0; p < npts; p++) {
      for (int c = 0; c < h.ncomp; c++)
        fprintf(f, c + 1 < h.ncomp ? "%.9g " : "%.9g\n", h.values[p * h.ncomp + c]);
    }
  }
  fclose(f);
}

// Live writers, for the final-state files written at upcxx::finalize()
std::set<Writer*>& live_writers() {
  static std::set<Writer*> w;
  return w;
}

}  // namespace

extern "C" void sns_api_finalize_hooks(void) {
  // finalize() is also reached from the error exit of the API; run once
  static bool ran = false;
  const char* prefix = getenv("SNS_WRITER_FINAL");
  if (ran || !prefix || !prefix[0]) return;
  ran = true;
  for (Writer* w : live_writers())
    if (w->fields() > 0) w->writeFile(string(prefix) + w->name() + ".vtk");
}

Writer::Writer(string name) : m_name(name), m_count(0), m_writes(0), m_f(1) {
  live_writers().insert(this);
}

Writer::~Writer() {
  live_writers().erase(this);
  wait_pending();
  if (m_out.is_open()) m_out.close();
}

void Writer::wait_pending() {
  if (m_job.joinable()) m_job.join();
}

void Writer::add(Scalar& a_scalar, string a_name) {
  m_scalars.push_back(&a_scalar);
  m_scalar_names.push_back(a_name);
}

void Writer::add(Vector& a_vector, string a_name) {
  m_vectors.push_back(&a_vector);
  m_vector_names.push_back(a_name);
}

void Writer::setFreq(int a_f) { m_f = a_f; }

// Physical values of the registered fields on the host now (the caller may
// change the fields as soon as this returns): scalars first, then vectors.
std::shared_ptr<vector<SnsWriterField>> Writer::collect(array<INT, DIM>& dims,
                                                   array<INT, DIM>& pdims) const {
  const size_t ns = m_scalars.size(), nv = m_vectors.size();
  if (ns + nv == 0) SNS_API_ERROR("variables list is empty");
  dims = ns ? m_scalars[0]->getDims() : m_vectors[0]->getDims();
  pdims = ns ? m_scalars[0]->getPDims() : m_vectors[0]->getPDims();
  const INT npts = pdims[0] * pdims[1] * pdims[2];
  auto fields = std::make_shared<vector<SnsWriterField>>();
  for (size_t i = 0; i < ns; i++) {
    SnsWriterField h{m_scalar_names[i], 1, vector<float>(npts)};
    if (m_scalars[i]->isFourier()) {
      Scalar tmp;
      m_scalars[i]->inverse(tmp);
      real_parts(tmp, h.values.data(), 1);
    } else {
      real_parts(*m_scalars[i], h.values.data(), 1);
    }
    fields->push_back(std::move(h));
  }
  for (size_t i = 0; i < nv; i++) {
    SnsWriterField h{m_vector_names[i], DIM, vector<float>(DIM * npts)};
    if (m_vectors[i]->isFourier()) {
      Vector tmp;
      m_vectors[i]->inverse(tmp);
      for (int d = 0; d < DIM; d++) real_parts(tmp[d], h.values.data() + d, DIM);
    } else {
      for (int d = 0; d < DIM; d++) real_parts((*m_vectors[i])[d], h.values.data() + d, DIM);
    }
    fields->push_back(std::move(h));
  }
  return fields;
}

void Writer::write() {
#ifndef NWRITE
  // the reference computes m_count++ % m_f (src/Writer.cpp:39), which faults
  // for the m_f = 0 that exec/ns.cpp sets; a frequency <= 0 writes nothing
  if (m_f <= 0) {
    m_count++;
    return;
  }
  if (m_count++ % m_f != 0) return;
  array<INT, DIM> dims, pdims;
  auto fields = collect(dims, pdims);
  const string fname = m_name + "0_" + to_string(m_writes++) + ".vtk";
  if (!m_out.is_open()) {
    m_out.open(m_name + ".visit");
    m_out << "!NBLOCKS " << upcxx::rank_n() << endl;
  }
  m_out << fname << endl;
  // format and write in the background; one file in flight
  wait_pending();
  m_job = thread([fname, dims, pdims, fields]() { write_vtk(fname, dims, pdims, *fields); });
#endif
}

void Writer::writeFile(const string& fname) {
  array<INT, DIM> dims, pdims;
  auto fields = collect(dims, pdims);
  wait_pending();
  write_vtk(fname, dims, pdims, *fields);
}
