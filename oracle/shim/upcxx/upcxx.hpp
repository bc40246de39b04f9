// TEST INFRASTRUCTURE ONLY -- single-rank stand-in for the UPC++ API, used to
// compile the reference's own sources (src/Scalar.cpp, src/Vector.cpp, ...)
// in place for the CPU oracle.  UPC++ itself is not installed here.  Only the
// calls the reference makes exist (src/Scalar.cpp:26-124, 135, 147, 454-626;
// exec/ns.cpp:28-229; exec/fft.cpp:30-91): with one rank every global pointer
// is local, broadcast returns its argument, rput/rget are copies and futures
// are always ready.
#ifndef ORACLE_UPCXX_STUB_HPP
#define ORACLE_UPCXX_STUB_HPP

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <utility>

namespace upcxx {

inline void init() {}
inline void finalize() {}
inline int rank_me() { return 0; }
inline int rank_n() { return 1; }
inline void barrier() {}

template <typename T>
class global_ptr {
 public:
  global_ptr() : p_(nullptr) {}
  global_ptr(std::nullptr_t) : p_(nullptr) {}
  explicit global_ptr(T* p) : p_(p) {}
  T* local() const { return p_; }
  global_ptr operator+(std::ptrdiff_t d) const { return global_ptr(p_ + d); }
  global_ptr operator+(std::size_t d) const { return global_ptr(p_ + d); }
  global_ptr operator+(int d) const { return global_ptr(p_ + d); }
  global_ptr operator+(long long d) const { return global_ptr(p_ + d); }
  global_ptr operator+(unsigned long long d) const { return global_ptr(p_ + d); }
  bool operator==(std::nullptr_t) const { return p_ == nullptr; }
  bool operator!=(std::nullptr_t) const { return p_ != nullptr; }
  bool operator==(const global_ptr& o) const { return p_ == o.p_; }
  bool operator!=(const global_ptr& o) const { return p_ != o.p_; }
  bool is_null() const { return p_ == nullptr; }
  int where() const { return 0; }

 private:
  T* p_;
};

template <typename... T>
class future;

template <>
class future<> {
 public:
  void wait() const {}
  bool ready() const { return true; }
};

template <typename T>
class future<T> {
 public:
  explicit future(T v) : v_(std::move(v)) {}
  T wait() const { return v_; }
  bool ready() const { return true; }

 private:
  T v_;
};

inline future<> make_future() { return future<>(); }
template <typename T>
future<T> make_future(T v) {
  return future<T>(std::move(v));
}
inline future<> when_all(const future<>&, const future<>&) { return future<>(); }

template <typename T>
global_ptr<T> new_array(std::size_t n) {
  // value-initialised, as upcxx::new_array constructs each element
  return global_ptr<T>(new T[n]());
}
template <typename T>
void delete_array(global_ptr<T> p) {
  delete[] p.local();
}
template <typename T, typename... Args>
global_ptr<T> new_(Args&&... args) {
  return global_ptr<T>(new T(std::forward<Args>(args)...));
}
template <typename T>
void delete_(global_ptr<T> p) {
  delete p.local();
}

template <typename T>
future<T> broadcast(T v, int /*root*/) {
  return future<T>(std::move(v));
}

template <typename T>
future<> rput(T v, global_ptr<T> dst) {
  *dst.local() = v;
  return future<>();
}
template <typename T>
future<> rput(const T* src, global_ptr<T> dst, std::size_t n) {
  std::memcpy((void*)dst.local(), (const void*)src, n * sizeof(T));
  return future<>();
}
template <typename T>
future<T> rget(global_ptr<T> src) {
  return future<T>(*src.local());
}

template <typename T, typename Op>
future<T> allreduce(T v, Op) {
  return future<T>(v);
}

struct persona_scope {};
inline persona_scope default_persona_scope() { return persona_scope(); }

}  // namespace upcxx

#endif
