// TEST INFRASTRUCTURE ONLY -- stand-in for owl::common, so that the
// reference's own hot-path headers and sources compile here from where they
// lie, unmodified, into oracle/_ref (see oracle/Makefile, target `ref`).
//
// OWL 1.2.9 (the version the reference's CMakeLists.txt:27 pins) is a git
// submodule that is not vendored with the reference.  This header defines the
// small part of its math library that the compiled reference files use, from
// the operations' mathematical meaning:
//   * vec_t<T,N>: N-component vectors with component-wise arithmetic,
//     scalar broadcast on either side, conversions between element types
//     (static_cast per component) and indexing;
//   * min / max: the smaller / larger operand by `<`, as written
//     (`a < b ? a : b`); clamp(x, lo, hi) = min(max(x, lo), hi);
//   * rcp(x) = 1/x, abs, reduce_min / reduce_max / arg_min over components;
//   * interval<T>: [lower, upper], empty by default (+inf, -inf), extend()
//     and span() = upper - lower;
//   * box_t: lower / upper corners.
// Nothing here is copied from OWL; only the names follow it, because the
// reference's sources call them by these names.
#pragma once

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#define OWL_ALIGN(a) alignas(a)
#ifndef __both__
#define __both__
#endif
#define PING fprintf(stderr, "%s:%d\n", __FILE__, __LINE__)
#define PRINT(x)

namespace owl {
namespace common {

using std::isnan;
using std::isinf;
using std::sqrt;

template <typename T>
inline T min(T a, T b) { return a < b ? a : b; }
template <typename T>
inline T max(T a, T b) { return a > b ? a : b; }
template <typename T>
inline T clamp(T x, T lo, T hi) { return min(max(x, lo), hi); }
inline float rcp(float x) { return 1.f / x; }

template <typename T, int N>
struct vec_t;

template <typename T>
struct vec_t<T, 2> {
  T x, y;
  vec_t() = default;
  vec_t(T s) : x(s), y(s) {}
  vec_t(T a, T b) : x(a), y(b) {}
  template <typename U>
  explicit vec_t(const vec_t<U, 2> &o) : x(T(o.x)), y(T(o.y)) {}
  T &operator[](int i) { return (&x)[i]; }
  T operator[](int i) const { return (&x)[i]; }
};
template <typename T>
struct vec_t<T, 3> {
  T x, y, z;
  vec_t() = default;
  vec_t(T s) : x(s), y(s), z(s) {}
  vec_t(T a, T b, T c) : x(a), y(b), z(c) {}
  template <typename U>
  explicit vec_t(const vec_t<U, 3> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
  T &operator[](int i) { return (&x)[i]; }
  T operator[](int i) const { return (&x)[i]; }
};
template <typename T>
struct vec_t<T, 4> {
  T x, y, z, w;
  vec_t() = default;
  vec_t(T s) : x(s), y(s), z(s), w(s) {}
  vec_t(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
  vec_t(const vec_t<T, 3> &v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
  template <typename U>
  explicit vec_t(const vec_t<U, 4> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)), w(T(o.w)) {}
  // a scalar of another type broadcast (vec4f(unsigned char))
  template <typename U, typename = typename std::enable_if<std::is_arithmetic<U>::value &&
                                                           !std::is_same<U, T>::value>::type>
  explicit vec_t(U s) : x(T(s)), y(T(s)), z(T(s)), w(T(s)) {}
  T &operator[](int i) { return (&x)[i]; }
  T operator[](int i) const { return (&x)[i]; }
};

using vec2f = vec_t<float, 2>;
using vec2i = vec_t<int, 2>;
using vec3f = vec_t<float, 3>;
using vec3i = vec_t<int, 3>;
using vec3ui = vec_t<uint32_t, 3>;
using vec4f = vec_t<float, 4>;
using vec4i = vec_t<int, 4>;
using vec4uc = vec_t<uint8_t, 4>;

#define BNREF_VEC_BINOP(OP)                                                                          \
  template <typename T>                                                                              \
  inline vec_t<T, 2> operator OP(const vec_t<T, 2> &a, const vec_t<T, 2> &b) {                       \
    return vec_t<T, 2>(a.x OP b.x, a.y OP b.y);                                                      \
  }                                                                                                  \
  template <typename T>                                                                              \
  inline vec_t<T, 3> operator OP(const vec_t<T, 3> &a, const vec_t<T, 3> &b) {                       \
    return vec_t<T, 3>(a.x OP b.x, a.y OP b.y, a.z OP b.z);                                          \
  }                                                                                                  \
  template <typename T>                                                                              \
  inline vec_t<T, 4> operator OP(const vec_t<T, 4> &a, const vec_t<T, 4> &b) {                       \
    return vec_t<T, 4>(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w);                              \
  }                                                                                                  \
  template <typename T, int N>                                                                       \
  inline vec_t<T, N> operator OP(const vec_t<T, N> &a, T s) { return a OP vec_t<T, N>(s); }          \
  template <typename T, int N>                                                                       \
  inline vec_t<T, N> operator OP(T s, const vec_t<T, N> &a) { return vec_t<T, N>(s) OP a; }          \
  template <typename T, int N>                                                                       \
  inline vec_t<T, N> &operator OP##=(vec_t<T, N> &a, const vec_t<T, N> &b) { return a = a OP b; }  \
  template <typename T, int N>                                                                       \
  inline vec_t<T, N> &operator OP##=(vec_t<T, N> &a, T s) { return a = a OP vec_t<T, N>(s); }

BNREF_VEC_BINOP(+)
BNREF_VEC_BINOP(-)
BNREF_VEC_BINOP(*)
BNREF_VEC_BINOP(/)
#undef BNREF_VEC_BINOP

template <typename T>
inline vec_t<T, 3> operator-(const vec_t<T, 3> &a) { return vec_t<T, 3>(-a.x, -a.y, -a.z); }
template <typename T>
inline vec_t<T, 4> operator-(const vec_t<T, 4> &a) { return vec_t<T, 4>(-a.x, -a.y, -a.z, -a.w); }
template <typename T>
inline bool operator==(const vec_t<T, 3> &a, const vec_t<T, 3> &b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
template <typename T>
inline bool operator!=(const vec_t<T, 3> &a, const vec_t<T, 3> &b) { return !(a == b); }

template <typename T>
inline vec_t<T, 3> min(const vec_t<T, 3> &a, const vec_t<T, 3> &b) {
  return vec_t<T, 3>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z));
}
template <typename T>
inline vec_t<T, 3> max(const vec_t<T, 3> &a, const vec_t<T, 3> &b) {
  return vec_t<T, 3>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z));
}
template <typename T>
inline vec_t<T, 4> min(const vec_t<T, 4> &a, const vec_t<T, 4> &b) {
  return vec_t<T, 4>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z), min(a.w, b.w));
}
template <typename T>
inline vec_t<T, 4> max(const vec_t<T, 4> &a, const vec_t<T, 4> &b) {
  return vec_t<T, 4>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z), max(a.w, b.w));
}
template <typename T>
inline T reduce_min(const vec_t<T, 3> &a) { return min(min(a.x, a.y), a.z); }
template <typename T>
inline T reduce_max(const vec_t<T, 3> &a) { return max(max(a.x, a.y), a.z); }
template <typename T>
inline T reduce_max(const vec_t<T, 4> &a) { return max(max(max(a.x, a.y), a.z), a.w); }
// index of the smallest component (the first one on ties)
template <typename T>
inline int arg_min(const vec_t<T, 3> &a) {
  return (a.x <= a.y && a.x <= a.z) ? 0 : (a.y <= a.z ? 1 : 2);
}
inline vec3f rcp(const vec3f &a) { return vec3f(1.f / a.x, 1.f / a.y, 1.f / a.z); }
inline float abs(float a) { return std::fabs(a); }
inline vec3f abs(const vec3f &a) { return vec3f(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
inline float dot(const vec3f &a, const vec3f &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3f cross(const vec3f &a, const vec3f &b) {
  return vec3f(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(const vec3f &a) { return std::sqrt(dot(a, a)); }
inline vec3f normalize(const vec3f &a) { return a * (1.f / std::sqrt(dot(a, a))); }

template <typename T>
struct interval {
  T lower = std::numeric_limits<T>::infinity();
  T upper = -std::numeric_limits<T>::infinity();
  interval() = default;
  interval(T lo, T hi) : lower(lo), upper(hi) {}
  T span() const { return upper - lower; }
  bool empty() const { return upper < lower; }
  interval &extend(T v) {
    lower = min(lower, v);
    upper = max(upper, v);
    return *this;
  }
};

template <typename V>
struct box_t {
  V lower, upper;
  box_t() = default;
  box_t(const V &lo, const V &hi) : lower(lo), upper(hi) {}
};
using box3f = box_t<vec3f>;
using box4f = box_t<vec4f>;

}  // namespace common
}  // namespace owl
