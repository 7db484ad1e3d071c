// Minimal stand-in for the dlib matrix type used by frame-aligner's FrameWarper.h and
// OptimisationModel.cpp (TEST INFRASTRUCTURE ONLY; lets the reference sources compile unchanged).
// Only storage and element access are provided: the trust-region solver is not part of this
// stand-in (the oracle's own solver drives the reference warper instead).
#pragma once
#include <cstddef>
#include <vector>

namespace dlib {

template <typename T, long NR = 0, long NC = 0>
class matrix {
 public:
  typedef T type;
  matrix() {}
  explicit matrix(long n) { set_size(n); }
  void set_size(long n) { nr_ = n; nc_ = 1; d_.assign((size_t)n, T()); }
  void set_size(long r, long c) { nr_ = r; nc_ = c; d_.assign((size_t)(r * c), T()); }
  T& operator()(long i) { return d_[(size_t)i]; }
  const T& operator()(long i) const { return d_[(size_t)i]; }
  T& operator()(long r, long c) { return d_[(size_t)(r * nc_ + c)]; }
  const T& operator()(long r, long c) const { return d_[(size_t)(r * nc_ + c)]; }
  typename std::vector<T>::iterator begin() { return d_.begin(); }
  typename std::vector<T>::iterator end() { return d_.end(); }
  typename std::vector<T>::const_iterator begin() const { return d_.begin(); }
  typename std::vector<T>::const_iterator end() const { return d_.end(); }
  long size() const { return (long)d_.size(); }
  long nr() const { return nr_; }
  long nc() const { return nc_; }
  T* data() { return d_.data(); }
  const T* data() const { return d_.data(); }

 private:
  std::vector<T> d_;
  long nr_ = 0, nc_ = 0;
};

}  // namespace dlib
