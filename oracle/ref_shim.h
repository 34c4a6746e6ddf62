// ref_shim.h -- the few Loci types that flowPsi's face functions use
// (vector3d, Array, Mat), so those functions compile from their own source
// for the oracle's cross-check.  Test infrastructure only.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>

namespace Loci {
template <class T>
struct vector3d {
  T x, y, z;
  vector3d() {}
  vector3d(T a, T b, T c) : x(a), y(b), z(c) {}
};
template <class T> inline vector3d<T> operator+(const vector3d<T>& a, const vector3d<T>& b) {
  return vector3d<T>(a.x + b.x, a.y + b.y, a.z + b.z);
}
template <class T> inline vector3d<T> operator-(const vector3d<T>& a, const vector3d<T>& b) {
  return vector3d<T>(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <class T> inline vector3d<T> operator*(const vector3d<T>& a, T s) {
  return vector3d<T>(a.x * s, a.y * s, a.z * s);
}
template <class T> inline vector3d<T> operator*(T s, const vector3d<T>& a) {
  return vector3d<T>(s * a.x, s * a.y, s * a.z);
}
template <class T> inline vector3d<T> operator/(const vector3d<T>& a, T s) {
  return vector3d<T>(a.x / s, a.y / s, a.z / s);
}
template <class T> inline T dot(const vector3d<T>& a, const vector3d<T>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T, size_t n>
struct Array {
  T d[n];
  T& operator[](size_t i) { return d[i]; }
  const T& operator[](size_t i) const { return d[i]; }
};
template <class T>
struct Mat {
  T* p;
  int n;
  Mat(T* p_, int n_) : p(p_), n(n_) {}
  T* operator[](int i) const { return p + i * n; }
};
}  // namespace Loci

namespace flowPsi {
typedef double real;
typedef float real_fj;
typedef Loci::vector3d<real> vect3d;
using Loci::dot;
using Loci::Mat;
using std::abs;
using std::fabs;
using std::max;
using std::min;
using std::sqrt;
}  // namespace flowPsi
