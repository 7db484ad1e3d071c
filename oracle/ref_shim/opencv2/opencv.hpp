// Minimal stand-in for the subset of OpenCV 4 that frame-aligner's warper path uses
// (FrameWarper.h/.cpp, Sobel3d.cpp, VolumePhaseCorrelator.h/.cpp, OptimisationModel.cpp).
//
// TEST INFRASTRUCTURE ONLY. It exists so that the reference's own source files compile
// unchanged with g++ (oracle/Makefile, target _ref/libfa_ref.so) and can be used to pin the
// oracle. It is written for this project from the OpenCV documentation of the members used:
// n-dimensional continuous Mat with reference-counted storage, at<T>(i0,i1,i2), size[],
// copyTo, convertTo (saturate + round-to-nearest), element-wise subtraction, Point3_ arithmetic.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <limits>
#include <iostream>
#include <algorithm>

#define CV_8U 0
#define CV_16U 2
#define CV_32F 5
#define CV_64F 6

namespace cv {

typedef unsigned char uchar;

template <typename T>
class Point3_ {
 public:
  Point3_() : x(0), y(0), z(0) {}
  Point3_(T x_, T y_, T z_) : x(x_), y(y_), z(z_) {}
  template <typename U>
  explicit Point3_(const Point3_<U>& o) : x((T)o.x), y((T)o.y), z((T)o.z) {}
  Point3_& operator+=(const Point3_& o) { x += o.x; y += o.y; z += o.z; return *this; }
  Point3_& operator-=(const Point3_& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  Point3_& operator*=(double s) { x = (T)(x * s); y = (T)(y * s); z = (T)(z * s); return *this; }
  T x, y, z;
};
template <typename T> inline Point3_<T> operator+(const Point3_<T>& a, const Point3_<T>& b) { return Point3_<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> inline Point3_<T> operator-(const Point3_<T>& a, const Point3_<T>& b) { return Point3_<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> inline Point3_<T> operator*(double s, const Point3_<T>& a) { return Point3_<T>((T)(s * a.x), (T)(s * a.y), (T)(s * a.z)); }
template <typename T> inline Point3_<T> operator*(const Point3_<T>& a, double s) { return s * a; }

typedef Point3_<int> Point3i;
typedef Point3_<float> Point3f;
typedef Point3_<double> Point3d;

template <typename T, int n>
class Vec {
 public:
  T v[n];
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
};

class Scalar {
 public:
  Scalar(double v0 = 0) : val{v0, 0, 0, 0} {}
  double operator[](int i) const { return val[i]; }
  double val[4];
};

inline size_t elemSizeOf(int type) {
  switch (type) {
    case CV_8U: return 1;
    case CV_16U: return 2;
    case CV_32F: return 4;
    case CV_64F: return 8;
  }
  throw std::runtime_error("shim Mat: unsupported type");
}

class MatSize {
 public:
  int operator[](int i) const { return p[i]; }
  int& operator[](int i) { return p[i]; }
  operator const int*() const { return p; }
  int p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

class Mat {
 public:
  Mat() {}
  Mat(const std::vector<int>& sizes, int type) { create(sizes, type); }
  Mat(const std::vector<int>& sizes, int type, const Scalar& s) { create(sizes, type); setTo(s[0]); }
  Mat(int ndims, const int* sizes, int type) { create(std::vector<int>(sizes, sizes + ndims), type); }

  void create(const std::vector<int>& sizes, int type) {
    dims = (int)sizes.size();
    type_ = type;
    size_t n = 1;
    for (int i = 0; i < dims; i++) { size[i] = sizes[i]; n *= (size_t)sizes[i]; }
    total_ = n;
    buf_ = std::shared_ptr<std::vector<uchar>>(new std::vector<uchar>(n * elemSizeOf(type) + 16, 0));
    data = buf_->data();
    step_[dims - 1] = elemSizeOf(type);
    for (int i = dims - 2; i >= 0; i--) step_[i] = step_[i + 1] * (size_t)size[i + 1];
  }

  void setTo(double v) {
    for (size_t i = 0; i < total_; i++) storeAs(i, v);
  }

  template <typename T>
  T& at(int i0, int i1, int i2) {
    return *reinterpret_cast<T*>(data + step_[0] * (size_t)i0 + step_[1] * (size_t)i1 + step_[2] * (size_t)i2);
  }
  template <typename T>
  const T& at(int i0, int i1, int i2) const {
    return *reinterpret_cast<const T*>(data + step_[0] * (size_t)i0 + step_[1] * (size_t)i1 + step_[2] * (size_t)i2);
  }
  template <typename T>
  T& at(int i) { return reinterpret_cast<T*>(data)[i]; }
  template <typename T>
  const T& at(int i) const { return reinterpret_cast<const T*>(data)[i]; }

  int type() const { return type_; }
  size_t elemSize() const { return elemSizeOf(type_); }
  size_t total() const { return total_; }
  bool empty() const { return data == nullptr || total_ == 0; }
  bool isContinuous() const { return true; }  // this stand-in only holds dense storage

  Mat clone() const {
    Mat m;
    if (empty()) return m;
    m.create(sizes(), type_);
    std::memcpy(m.data, data, total_ * elemSize());
    return m;
  }

  void copyTo(Mat& out) const {
    if (out.data == data) return;
    if (out.empty() || out.dims != dims || out.type_ != type_ || out.total_ != total_ || out.sizes() != sizes())
      out.create(sizes(), type_);
    std::memcpy(out.data, data, total_ * elemSize());
  }

  // Element conversion with OpenCV's saturate_cast semantics (round half to even via
  // std::nearbyint under the default rounding mode, then clamp) for integer targets.
  void convertTo(Mat& out, int rtype) const {
    Mat tmp;
    tmp.create(sizes(), rtype);
    for (size_t i = 0; i < total_; i++) tmp.storeAs(i, loadAs(i));
    out = tmp;
  }

  std::vector<int> sizes() const { return std::vector<int>(size.p, size.p + dims); }

  double loadAs(size_t i) const {
    switch (type_) {
      case CV_8U: return reinterpret_cast<const uint8_t*>(data)[i];
      case CV_16U: return reinterpret_cast<const uint16_t*>(data)[i];
      case CV_32F: return reinterpret_cast<const float*>(data)[i];
      case CV_64F: return reinterpret_cast<const double*>(data)[i];
    }
    return 0;
  }
  void storeAs(size_t i, double v) {
    switch (type_) {
      case CV_8U: { double r = std::nearbyint(v); r = std::min(255.0, std::max(0.0, r)); if (v != v) r = 0; reinterpret_cast<uint8_t*>(data)[i] = (uint8_t)r; break; }
      case CV_16U: { double r = std::nearbyint(v); r = std::min(65535.0, std::max(0.0, r)); if (v != v) r = 0; reinterpret_cast<uint16_t*>(data)[i] = (uint16_t)r; break; }
      case CV_32F: reinterpret_cast<float*>(data)[i] = (float)v; break;
      case CV_64F: reinterpret_cast<double*>(data)[i] = v; break;
    }
  }

  int dims = 0;
  uchar* data = nullptr;
  MatSize size;

 private:
  int type_ = CV_32F;
  size_t total_ = 0;
  size_t step_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::shared_ptr<std::vector<uchar>> buf_;
};

// Element-wise difference of two CV_32F matrices, computed in float as OpenCV does for
// same-type float operands.
inline Mat operator-(const Mat& a, const Mat& b) {
  if (a.type() != CV_32F || b.type() != CV_32F || a.total() != b.total())
    throw std::runtime_error("shim Mat: subtraction needs equal-size CV_32F operands");
  Mat r(a.sizes(), CV_32F);
  const float* pa = reinterpret_cast<const float*>(a.data);
  const float* pb = reinterpret_cast<const float*>(b.data);
  float* pr = reinterpret_cast<float*>(r.data);
  for (size_t i = 0; i < a.total(); i++) pr[i] = pa[i] - pb[i];
  return r;
}

}  // namespace cv
