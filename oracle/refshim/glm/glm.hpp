// Minimal stand-in for the parts of glm the reference's FluidSim CPU path uses
// (used only to build the reference's own sources into oracle/_ref): small
// fixed-size vectors with component-wise IEEE arithmetic, dot, length,
// distance, normalize and clamp.  Matrix types are declared only.
#pragma once
#include <cmath>
#include <cstddef>
namespace glm {
enum qualifier { defaultp = 0 };
template <int N, class T, qualifier Q = defaultp> struct vec;
template <class T, qualifier Q> struct vec<2, T, Q> {
  T x, y;
  vec() : x(0), y(0) {}
  explicit vec(T s) : x(s), y(s) {}
  vec(T a, T b) : x(a), y(b) {}
  template <class U> explicit vec(const vec<2, U, Q>& o) : x(T(o.x)), y(T(o.y)) {}
  T& operator[](int i) { return i == 0 ? x : y; }
  const T& operator[](int i) const { return i == 0 ? x : y; }
  static constexpr int length() { return 2; }
};
template <class T, qualifier Q> struct vec<3, T, Q> {
  T x, y, z;
  vec() : x(0), y(0), z(0) {}
  explicit vec(T s) : x(s), y(s), z(s) {}
  vec(T a, T b, T c) : x(a), y(b), z(c) {}
  template <class U> explicit vec(const vec<3, U, Q>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
  T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  static constexpr int length() { return 3; }
};
template <class T, qualifier Q> struct vec<4, T, Q> {
  T x, y, z, w;
  vec() : x(0), y(0), z(0), w(0) {}
  explicit vec(T s) : x(s), y(s), z(s), w(s) {}
  vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
  T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  static constexpr int length() { return 4; }
};
#define GLMS_BIN(OP)                                                                   \
  template <int N, class T, qualifier Q>                                               \
  vec<N, T, Q> operator OP(const vec<N, T, Q>& a, const vec<N, T, Q>& b) {             \
    vec<N, T, Q> r;                                                                    \
    for (int i = 0; i < N; i++) r[i] = a[i] OP b[i];                                   \
    return r;                                                                          \
  }                                                                                    \
  template <int N, class T, qualifier Q>                                               \
  vec<N, T, Q> operator OP(const vec<N, T, Q>& a, T s) {                               \
    vec<N, T, Q> r;                                                                    \
    for (int i = 0; i < N; i++) r[i] = a[i] OP s;                                      \
    return r;                                                                          \
  }                                                                                    \
  template <int N, class T, qualifier Q>                                               \
  vec<N, T, Q> operator OP(T s, const vec<N, T, Q>& a) {                               \
    vec<N, T, Q> r;                                                                    \
    for (int i = 0; i < N; i++) r[i] = s OP a[i];                                      \
    return r;                                                                          \
  }                                                                                    \
  template <int N, class T, qualifier Q>                                               \
  vec<N, T, Q>& operator OP##=(vec<N, T, Q>& a, const vec<N, T, Q>& b) {               \
    for (int i = 0; i < N; i++) a[i] = a[i] OP b[i];                                   \
    return a;                                                                          \
  }                                                                                    \
  template <int N, class T, qualifier Q>                                               \
  vec<N, T, Q>& operator OP##=(vec<N, T, Q>& a, T s) {                                 \
    for (int i = 0; i < N; i++) a[i] = a[i] OP s;                                      \
    return a;                                                                          \
  }
GLMS_BIN(+)
GLMS_BIN(-)
GLMS_BIN(*)
GLMS_BIN(/)
#undef GLMS_BIN
template <int N, class T, qualifier Q> vec<N, T, Q> operator-(const vec<N, T, Q>& a) {
  vec<N, T, Q> r;
  for (int i = 0; i < N; i++) r[i] = -a[i];
  return r;
}
template <int N, class T, qualifier Q> bool operator==(const vec<N, T, Q>& a, const vec<N, T, Q>& b) {
  for (int i = 0; i < N; i++)
    if (!(a[i] == b[i])) return false;
  return true;
}
template <int N, class T, qualifier Q> bool operator!=(const vec<N, T, Q>& a, const vec<N, T, Q>& b) {
  return !(a == b);
}
// dot: products first, then summed left to right
template <int N, class T, qualifier Q> T dot(const vec<N, T, Q>& a, const vec<N, T, Q>& b) {
  vec<N, T, Q> p = a * b;
  T s = p[0];
  for (int i = 1; i < N; i++) s = s + p[i];
  return s;
}
template <int N, class T, qualifier Q> T length(const vec<N, T, Q>& a) { return std::sqrt(dot(a, a)); }
template <int N, class T, qualifier Q> T distance(const vec<N, T, Q>& a, const vec<N, T, Q>& b) {
  return length(b - a);
}
// normalize: x * (1 / sqrt(x . x))
template <int N, class T, qualifier Q> vec<N, T, Q> normalize(const vec<N, T, Q>& a) {
  return a * (T(1) / std::sqrt(dot(a, a)));
}
template <class T> T clamp(T x, T lo, T hi) { return std::fmin(std::fmax(x, lo), hi); }
template <int N, class T, qualifier Q> vec<N, T, Q> clamp(const vec<N, T, Q>& x, T lo, T hi) {
  vec<N, T, Q> r;
  for (int i = 0; i < N; i++) r[i] = clamp(x[i], lo, hi);
  return r;
}
template <class T> using tvec2 = vec<2, T>;
template <class T> using tvec3 = vec<3, T>;
template <class T> using tvec4 = vec<4, T>;
using vec2 = vec<2, float>; using vec3 = vec<3, float>; using vec4 = vec<4, float>;
using dvec2 = vec<2, double>; using dvec3 = vec<3, double>; using dvec4 = vec<4, double>;
using ivec2 = vec<2, int>; using ivec3 = vec<3, int>; using ivec4 = vec<4, int>;
using uvec2 = vec<2, unsigned>; using uvec3 = vec<3, unsigned>; using uvec4 = vec<4, unsigned>;
template <int C, int R, class T> struct mat { vec<R, T> col[C]; };
template <class T> using tmat2x2 = mat<2, 2, T>;
template <class T> using tmat3x3 = mat<3, 3, T>;
template <class T> using tmat4x4 = mat<4, 4, T>;
using mat2 = mat<2, 2, float>; using mat3 = mat<3, 3, float>; using mat4 = mat<4, 4, float>;
using highp_mat2 = mat2; using highp_mat3 = mat3; using highp_mat4 = mat4;
using dmat2 = mat<2, 2, double>; using dmat3 = mat<3, 3, double>; using dmat4 = mat<4, 4, double>;
}  // namespace glm
