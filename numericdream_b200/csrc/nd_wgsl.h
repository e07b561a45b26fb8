// WGSL value types and builtins for translated formula code (host and device).
//
// Translated formulas (numericdream_b200/translator/wgsl.py) are C++ function
// templates over the float type T.  This header gives them WGSL's vector, matrix
// and array types and the builtin functions with WGSL semantics:
//   * round() is round-half-to-even;  fract(x) = x - floor(x);  sign(0) = 0
//   * float->int conversion truncates and saturates (NaN -> 0)
//   * float % is x - y * trunc(x / y);  integer x / 0 = x and x % 0 = 0
//   * shifts use the shift amount modulo 32
//   * mix(a, b, t) = a * (1 - t) + b * t;  step(e, x) = x >= e ? 1 : 0
//   * pow(x, y) is NaN for x < 0 (the SPIR-V/MSL/HLSL pow leaves it undefined; the
//     formulas only use it on non-negative bases)
//   * every index is clamped into range, as WGSL's robust access allows
#pragma once

#include <stdint.h>
#include <math.h>
#include <string.h>

#include <type_traits>

#if defined(__CUDACC__)
#define ND_HD_INLINE __host__ __device__ __forceinline__
#define ND_HD __host__ __device__
#else
#define ND_HD_INLINE inline
#define ND_HD
#endif

namespace ndw {

// ---------------------------------------------------------------- polynomial acos / atan2
// f32 arccosine and two-argument arctangent as short polynomials, for the fast-math
// device build (acosf / atan2f are long range-reduced routines).  The coefficients
// were fitted for this library (least squares on 4000 Chebyshev nodes refined by
// Lawson's iteration toward the minimax fit):
//   acos(a) = sqrt(1 - a) * P(a) on [0, 1], P of degree 7, |error| <= 2.2e-8;
//   atan(a) = a * Q(a^2) on [0, 1], Q of degree 8, |error| <= 1.4e-8;
// the other octants by acos(-x) = pi - acos(x), atan(1/a) = pi/2 - atan(a),
// atan2(y, -x) = pi - atan2(y, x) and the sign of y.  Rounded in f32 they stay within
// a few ulp (tests/test_wgsl_math.py), far inside WGSL's accuracy rules for acos and
// atan2.  NaN arguments give NaN; atan2 of two infinities gives the octant angle.
ND_HD_INLINE float nd_acos_poly(float x) {
  const float a = fabsf(x);
  float p = -0.0012628166408258335f;
  p = fmaf(p, a, 0.006671243789107799f);
  p = fmaf(p, a, -0.017089743594000825f);
  p = fmaf(p, a, 0.030893008030167084f);
  p = fmaf(p, a, -0.0501746996877574f);
  p = fmaf(p, a, 0.08897904736598193f);
  p = fmaf(p, a, -0.21459880368099798f);
  p = fmaf(p, a, 1.5707963049937743f);
  const float r = sqrtf(1.0f - a) * p;
  // pi - r with pi split into an f32 head and tail
  return x < 0.0f ? (3.14159274f - r) + -8.74227766e-8f : r;
}

ND_HD_INLINE float nd_atan2_poly(float y, float x) {
  if (x != x || y != y) return x + y;
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  const float a = mx == mn ? (mx > 0.0f ? 1.0f : 0.0f) : mn / mx;
  const float s = a * a;
  float q = 0.0029035175208155816f;
  q = fmaf(q, s, -0.016282869281752363f);
  q = fmaf(q, s, 0.04303914484614859f);
  q = fmaf(q, s, -0.07533657424332961f);
  q = fmaf(q, s, 0.10654668786402743f);
  q = fmaf(q, s, -0.14207131502731904f);
  q = fmaf(q, s, 0.19993053843505385f);
  q = fmaf(q, s, -0.33333093945014514f);
  q = fmaf(q, s, 0.9999999863658048f);
  float r = a * q;
  if (ay > ax) r = (1.57079637f - r) + -4.37113883e-8f;
  if (copysignf(1.0f, x) < 0.0f) r = (3.14159274f - r) + -8.74227766e-8f;  // x < 0 or x = -0
  return copysignf(r, y);
}

#if defined(__CUDA_ARCH__) && !defined(ND_ACCURATE_MATH)
#define ND_ACOS_F(x) nd_acos_poly(x)
#define ND_ATAN2_F(y, x) nd_atan2_poly(y, x)
#else
#define ND_ACOS_F(x) acosf(x)
#define ND_ATAN2_F(y, x) atan2f(y, x)
#endif

// ---------------------------------------------------------------- scalars
#define ND_UNARY_F(NAME, FEXPR, DEXPR)                    \
  ND_HD_INLINE float NAME(float x) { return FEXPR; }      \
  ND_HD_INLINE double NAME(double x) { return DEXPR; }

ND_UNARY_F(sin, sinf(x), ::sin(x))
ND_UNARY_F(cos, cosf(x), ::cos(x))
ND_UNARY_F(tan, tanf(x), ::tan(x))
ND_UNARY_F(asin, asinf(x), ::asin(x))
ND_UNARY_F(acos, ND_ACOS_F(x), ::acos(x))
ND_UNARY_F(atan, atanf(x), ::atan(x))
ND_UNARY_F(sinh, sinhf(x), ::sinh(x))
ND_UNARY_F(cosh, coshf(x), ::cosh(x))
ND_UNARY_F(tanh, tanhf(x), ::tanh(x))
ND_UNARY_F(exp, expf(x), ::exp(x))
ND_UNARY_F(exp2, exp2f(x), ::exp2(x))
ND_UNARY_F(log, logf(x), ::log(x))
ND_UNARY_F(log2, log2f(x), ::log2(x))
ND_UNARY_F(sqrt, sqrtf(x), ::sqrt(x))
ND_UNARY_F(floor, floorf(x), ::floor(x))
ND_UNARY_F(ceil, ceilf(x), ::ceil(x))
ND_UNARY_F(trunc, truncf(x), ::trunc(x))
ND_UNARY_F(round, rintf(x), ::rint(x))
#undef ND_UNARY_F

ND_HD_INLINE float inverseSqrt(float x) { return 1.0f / sqrtf(x); }
ND_HD_INLINE double inverseSqrt(double x) { return 1.0 / ::sqrt(x); }
template <class T> ND_HD_INLINE T fract(T x) { return x - floor(x); }
ND_HD_INLINE float radians(float x) { return x * 0.017453292519943295f; }
ND_HD_INLINE double radians(double x) { return x * 0.017453292519943295; }
ND_HD_INLINE float degrees(float x) { return x * 57.29577951308232f; }
ND_HD_INLINE double degrees(double x) { return x * 57.29577951308232; }

ND_HD_INLINE float abs(float x) { return fabsf(x); }
ND_HD_INLINE double abs(double x) { return ::fabs(x); }
ND_HD_INLINE int32_t abs(int32_t x) { return x < 0 ? int32_t(0u - uint32_t(x)) : x; }
ND_HD_INLINE uint32_t abs(uint32_t x) { return x; }

ND_HD_INLINE float sign(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }
ND_HD_INLINE double sign(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }
ND_HD_INLINE int32_t sign(int32_t x) { return x > 0 ? 1 : (x < 0 ? -1 : 0); }

ND_HD_INLINE float min(float a, float b) { return fminf(a, b); }
ND_HD_INLINE double min(double a, double b) { return ::fmin(a, b); }
ND_HD_INLINE float max(float a, float b) { return fmaxf(a, b); }
ND_HD_INLINE double max(double a, double b) { return ::fmax(a, b); }
ND_HD_INLINE int32_t min(int32_t a, int32_t b) { return a < b ? a : b; }
ND_HD_INLINE int32_t max(int32_t a, int32_t b) { return a > b ? a : b; }
ND_HD_INLINE uint32_t min(uint32_t a, uint32_t b) { return a < b ? a : b; }
ND_HD_INLINE uint32_t max(uint32_t a, uint32_t b) { return a > b ? a : b; }

ND_HD_INLINE float pow(float x, float y) { return x < 0.0f ? __builtin_nanf("") : powf(x, y); }
ND_HD_INLINE double pow(double x, double y) { return x < 0.0 ? __builtin_nan("") : ::pow(x, y); }
ND_HD_INLINE float atan2(float y, float x) { return ND_ATAN2_F(y, x); }
ND_HD_INLINE double atan2(double y, double x) { return ::atan2(y, x); }
template <class T> ND_HD_INLINE T step(T edge, T x) { return x >= edge ? T(1) : T(0); }
template <class T> ND_HD_INLINE T clamp(T x, T lo, T hi) { return min(max(x, lo), hi); }
template <class T> ND_HD_INLINE T saturate(T x) { return clamp(x, T(0), T(1)); }
template <class T> ND_HD_INLINE T mix(T a, T b, T t) { return a * (T(1) - t) + b * t; }
template <class T> ND_HD_INLINE T smoothstep(T lo, T hi, T x) {
  T t = clamp((x - lo) / (hi - lo), T(0), T(1));
  return t * t * (T(3) - T(2) * t);
}
ND_HD_INLINE float fma(float a, float b, float c) { return fmaf(a, b, c); }
ND_HD_INLINE double fma(double a, double b, double c) { return ::fma(a, b, c); }
template <class T> ND_HD_INLINE T fmod_trunc(T a, T b) { return a - b * trunc(a / b); }

template <class T> ND_HD_INLINE T select(T f, T t, bool c) { return c ? t : f; }

// float -> integer conversions: truncate toward zero, saturate, NaN -> 0
template <class T> ND_HD_INLINE int32_t to_i32(T x) {
  double v = double(x);
  if (!(v == v)) return 0;
  if (v >= 2147483647.0) return 2147483647;
  if (v <= -2147483648.0) return int32_t(-2147483647 - 1);
  return int32_t(v);
}
template <class T> ND_HD_INLINE uint32_t to_u32(T x) {
  double v = double(x);
  if (!(v == v) || v <= 0.0) return 0u;
  if (v >= 4294967295.0) return 4294967295u;
  return uint32_t(v);
}
ND_HD_INLINE int32_t to_i32(float x) {
#if defined(__CUDA_ARCH__)
  return __float2int_rz(x);
#else
  if (!(x == x)) return 0;
  if (x >= 2147483647.0f) return 2147483647;
  if (x <= -2147483648.0f) return int32_t(-2147483647 - 1);
  return int32_t(x);
#endif
}
ND_HD_INLINE uint32_t to_u32(float x) {
#if defined(__CUDA_ARCH__)
  return __float2uint_rz(x);
#else
  if (!(x == x) || x <= 0.0f) return 0u;
  if (x >= 4294967295.0f) return 4294967295u;
  return uint32_t(x);
#endif
}

// bit casts go through the f32 representation (T may be wider than f32)
template <class T> ND_HD_INLINE uint32_t bitcast_u32(T x) {
  float f = float(x);
#if defined(__CUDA_ARCH__)
  return __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
#endif
}
template <class T> ND_HD_INLINE int32_t bitcast_i32(T x) { return int32_t(bitcast_u32(x)); }
ND_HD_INLINE float bitcast_f32(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
ND_HD_INLINE float bitcast_f32(int32_t i) { return bitcast_f32(uint32_t(i)); }

ND_HD_INLINE int32_t idiv(int32_t a, int32_t b) {
  if (b == 0) return a;
  if (a == int32_t(-2147483647 - 1) && b == -1) return a;
  return a / b;
}
ND_HD_INLINE uint32_t idiv(uint32_t a, uint32_t b) { return b == 0u ? a : a / b; }
ND_HD_INLINE int32_t irem(int32_t a, int32_t b) {
  if (b == 0) return 0;
  if (a == int32_t(-2147483647 - 1) && b == -1) return 0;
  return a % b;
}
ND_HD_INLINE uint32_t irem(uint32_t a, uint32_t b) { return b == 0u ? 0u : a % b; }
ND_HD_INLINE uint32_t shl(uint32_t a, uint32_t s) { return a << (s & 31u); }
ND_HD_INLINE uint32_t shr(uint32_t a, uint32_t s) { return a >> (s & 31u); }
ND_HD_INLINE int32_t shl(int32_t a, uint32_t s) { return int32_t(uint32_t(a) << (s & 31u)); }
ND_HD_INLINE int32_t shr(int32_t a, uint32_t s) { return a >> (s & 31u); }

ND_HD_INLINE uint32_t countOneBits(uint32_t x) {
#if defined(__CUDA_ARCH__)
  return __popc(x);
#else
  return uint32_t(__builtin_popcount(x));
#endif
}

// ---------------------------------------------------------------- vectors
template <class S> struct v2 {
  S x, y;
  ND_HD_INLINE v2() : x(S(0)), y(S(0)) {}
  ND_HD_INLINE explicit v2(S s) : x(s), y(s) {}
  ND_HD_INLINE v2(S a, S b) : x(a), y(b) {}
  ND_HD_INLINE S& operator[](int i) { return (i <= 0) ? x : y; }
  ND_HD_INLINE S operator[](int i) const { return (i <= 0) ? x : y; }
  ND_HD_INLINE S& operator[](uint32_t i) { return (*this)[int(i > 1u ? 1u : i)]; }
  ND_HD_INLINE S operator[](uint32_t i) const { return (*this)[int(i > 1u ? 1u : i)]; }
  static constexpr int N = 2;
};
template <class S> struct v3 {
  S x, y, z;
  ND_HD_INLINE v3() : x(S(0)), y(S(0)), z(S(0)) {}
  ND_HD_INLINE explicit v3(S s) : x(s), y(s), z(s) {}
  ND_HD_INLINE v3(S a, S b, S c) : x(a), y(b), z(c) {}
  ND_HD_INLINE v3(v2<S> a, S c) : x(a.x), y(a.y), z(c) {}
  ND_HD_INLINE v3(S a, v2<S> b) : x(a), y(b.x), z(b.y) {}
  ND_HD_INLINE S& operator[](int i) { return (i <= 0) ? x : (i == 1 ? y : z); }
  ND_HD_INLINE S operator[](int i) const { return (i <= 0) ? x : (i == 1 ? y : z); }
  ND_HD_INLINE S& operator[](uint32_t i) { return (*this)[int(i > 2u ? 2u : i)]; }
  ND_HD_INLINE S operator[](uint32_t i) const { return (*this)[int(i > 2u ? 2u : i)]; }
  static constexpr int N = 3;
};
template <class S> struct v4 {
  S x, y, z, w;
  ND_HD_INLINE v4() : x(S(0)), y(S(0)), z(S(0)), w(S(0)) {}
  ND_HD_INLINE explicit v4(S s) : x(s), y(s), z(s), w(s) {}
  ND_HD_INLINE v4(S a, S b, S c, S d) : x(a), y(b), z(c), w(d) {}
  ND_HD_INLINE v4(v3<S> a, S d) : x(a.x), y(a.y), z(a.z), w(d) {}
  ND_HD_INLINE v4(S a, v3<S> b) : x(a), y(b.x), z(b.y), w(b.z) {}
  ND_HD_INLINE v4(v2<S> a, v2<S> b) : x(a.x), y(a.y), z(b.x), w(b.y) {}
  ND_HD_INLINE v4(v2<S> a, S c, S d) : x(a.x), y(a.y), z(c), w(d) {}
  ND_HD_INLINE v4(S a, v2<S> b, S d) : x(a), y(b.x), z(b.y), w(d) {}
  ND_HD_INLINE v4(S a, S b, v2<S> c) : x(a), y(b), z(c.x), w(c.y) {}
  ND_HD_INLINE S& operator[](int i) { return (i <= 0) ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  ND_HD_INLINE S operator[](int i) const { return (i <= 0) ? x : (i == 1 ? y : (i == 2 ? z : w)); }
  ND_HD_INLINE S& operator[](uint32_t i) { return (*this)[int(i > 3u ? 3u : i)]; }
  ND_HD_INLINE S operator[](uint32_t i) const { return (*this)[int(i > 3u ? 3u : i)]; }
  static constexpr int N = 4;
};

// component-wise map helpers
#define ND_MAP1(V, EXPR) \
  V r;                   \
  for (int i = 0; i < V::N; ++i) r[i] = EXPR; \
  return r;

#define ND_VEC_BINOP(OP)                                                                          \
  template <class S> ND_HD_INLINE v2<S> operator OP(v2<S> a, v2<S> b) { return v2<S>(a.x OP b.x, a.y OP b.y); } \
  template <class S> ND_HD_INLINE v3<S> operator OP(v3<S> a, v3<S> b) { return v3<S>(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
  template <class S> ND_HD_INLINE v4<S> operator OP(v4<S> a, v4<S> b) { return v4<S>(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); } \
  template <class S> ND_HD_INLINE v2<S> operator OP(v2<S> a, S b) { return v2<S>(a.x OP b, a.y OP b); } \
  template <class S> ND_HD_INLINE v3<S> operator OP(v3<S> a, S b) { return v3<S>(a.x OP b, a.y OP b, a.z OP b); } \
  template <class S> ND_HD_INLINE v4<S> operator OP(v4<S> a, S b) { return v4<S>(a.x OP b, a.y OP b, a.z OP b, a.w OP b); } \
  template <class S> ND_HD_INLINE v2<S> operator OP(S a, v2<S> b) { return v2<S>(a OP b.x, a OP b.y); } \
  template <class S> ND_HD_INLINE v3<S> operator OP(S a, v3<S> b) { return v3<S>(a OP b.x, a OP b.y, a OP b.z); } \
  template <class S> ND_HD_INLINE v4<S> operator OP(S a, v4<S> b) { return v4<S>(a OP b.x, a OP b.y, a OP b.z, a OP b.w); }

ND_VEC_BINOP(+)
ND_VEC_BINOP(-)
ND_VEC_BINOP(*)
ND_VEC_BINOP(/)
ND_VEC_BINOP(&)
ND_VEC_BINOP(|)
ND_VEC_BINOP(^)
#undef ND_VEC_BINOP

template <class S> ND_HD_INLINE v2<S> operator-(v2<S> a) { return v2<S>(-a.x, -a.y); }
template <class S> ND_HD_INLINE v3<S> operator-(v3<S> a) { return v3<S>(-a.x, -a.y, -a.z); }
template <class S> ND_HD_INLINE v4<S> operator-(v4<S> a) { return v4<S>(-a.x, -a.y, -a.z, -a.w); }
template <class S> ND_HD_INLINE v2<S> operator~(v2<S> a) { return v2<S>(~a.x, ~a.y); }
template <class S> ND_HD_INLINE v3<S> operator~(v3<S> a) { return v3<S>(~a.x, ~a.y, ~a.z); }
template <class S> ND_HD_INLINE v4<S> operator~(v4<S> a) { return v4<S>(~a.x, ~a.y, ~a.z, ~a.w); }

template <class V, class U> ND_HD_INLINE V vshl_(V a, U s) { ND_MAP1(V, shl(a[i], s[i])) }
template <class V, class U> ND_HD_INLINE V vshr_(V a, U s) { ND_MAP1(V, shr(a[i], s[i])) }
template <class S> ND_HD_INLINE v2<S> shl(v2<S> a, v2<uint32_t> s) { return vshl_(a, s); }
template <class S> ND_HD_INLINE v3<S> shl(v3<S> a, v3<uint32_t> s) { return vshl_(a, s); }
template <class S> ND_HD_INLINE v4<S> shl(v4<S> a, v4<uint32_t> s) { return vshl_(a, s); }
template <class S> ND_HD_INLINE v2<S> shr(v2<S> a, v2<uint32_t> s) { return vshr_(a, s); }
template <class S> ND_HD_INLINE v3<S> shr(v3<S> a, v3<uint32_t> s) { return vshr_(a, s); }
template <class S> ND_HD_INLINE v4<S> shr(v4<S> a, v4<uint32_t> s) { return vshr_(a, s); }

template <class S> ND_HD_INLINE v2<S> idiv(v2<S> a, v2<S> b) { return v2<S>(idiv(a.x, b.x), idiv(a.y, b.y)); }
template <class S> ND_HD_INLINE v3<S> idiv(v3<S> a, v3<S> b) { return v3<S>(idiv(a.x, b.x), idiv(a.y, b.y), idiv(a.z, b.z)); }
template <class S> ND_HD_INLINE v2<S> irem(v2<S> a, v2<S> b) { return v2<S>(irem(a.x, b.x), irem(a.y, b.y)); }
template <class S> ND_HD_INLINE v3<S> irem(v3<S> a, v3<S> b) { return v3<S>(irem(a.x, b.x), irem(a.y, b.y), irem(a.z, b.z)); }

// comparisons -> bool vectors
#define ND_VCMP(NAME, OP)                                                                              \
  template <class S> ND_HD_INLINE v2<bool> NAME(v2<S> a, v2<S> b) { return v2<bool>(a.x OP b.x, a.y OP b.y); } \
  template <class S> ND_HD_INLINE v3<bool> NAME(v3<S> a, v3<S> b) { return v3<bool>(a.x OP b.x, a.y OP b.y, a.z OP b.z); } \
  template <class S> ND_HD_INLINE v4<bool> NAME(v4<S> a, v4<S> b) { return v4<bool>(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w); }
ND_VCMP(veq, ==)
ND_VCMP(vne, !=)
ND_VCMP(vlt, <)
ND_VCMP(vgt, >)
ND_VCMP(vle, <=)
ND_VCMP(vge, >=)
#undef ND_VCMP

template <class V> ND_HD_INLINE V vnot(V a) { ND_MAP1(V, !a[i]) }
template <class V> ND_HD_INLINE bool any(V a) {
  bool r = false;
  for (int i = 0; i < V::N; ++i) r = r || a[i];
  return r;
}
template <class V> ND_HD_INLINE bool all(V a) {
  bool r = true;
  for (int i = 0; i < V::N; ++i) r = r && a[i];
  return r;
}

template <int... I, class V> ND_HD_INLINE auto swz(V v) {
  using S = decltype(v.x);
  if constexpr (sizeof...(I) == 2) {
    constexpr int idx[2] = {I...};
    return v2<S>(v[idx[0]], v[idx[1]]);
  } else if constexpr (sizeof...(I) == 3) {
    constexpr int idx[3] = {I...};
    return v3<S>(v[idx[0]], v[idx[1]], v[idx[2]]);
  } else {
    constexpr int idx[4] = {I...};
    return v4<S>(v[idx[0]], v[idx[1]], v[idx[2]], v[idx[3]]);
  }
}

template <class D, class S> ND_HD_INLINE v2<D> vcast(v2<S> a) { return v2<D>(D(a.x), D(a.y)); }
template <class D, class S> ND_HD_INLINE v3<D> vcast(v3<S> a) { return v3<D>(D(a.x), D(a.y), D(a.z)); }
template <class D, class S> ND_HD_INLINE v4<D> vcast(v4<S> a) { return v4<D>(D(a.x), D(a.y), D(a.z), D(a.w)); }
template <class S> ND_HD_INLINE v2<int32_t> vto_i32(v2<S> a) { return v2<int32_t>(to_i32(a.x), to_i32(a.y)); }
template <class S> ND_HD_INLINE v3<int32_t> vto_i32(v3<S> a) { return v3<int32_t>(to_i32(a.x), to_i32(a.y), to_i32(a.z)); }
template <class S> ND_HD_INLINE v4<int32_t> vto_i32(v4<S> a) { return v4<int32_t>(to_i32(a.x), to_i32(a.y), to_i32(a.z), to_i32(a.w)); }
template <class S> ND_HD_INLINE v2<uint32_t> vto_u32(v2<S> a) { return v2<uint32_t>(to_u32(a.x), to_u32(a.y)); }
template <class S> ND_HD_INLINE v3<uint32_t> vto_u32(v3<S> a) { return v3<uint32_t>(to_u32(a.x), to_u32(a.y), to_u32(a.z)); }
template <class S> ND_HD_INLINE v4<uint32_t> vto_u32(v4<S> a) { return v4<uint32_t>(to_u32(a.x), to_u32(a.y), to_u32(a.z), to_u32(a.w)); }
template <class S> ND_HD_INLINE v2<uint32_t> vbitcast_u32(v2<S> a) { return v2<uint32_t>(bitcast_u32(a.x), bitcast_u32(a.y)); }
template <class S> ND_HD_INLINE v3<uint32_t> vbitcast_u32(v3<S> a) { return v3<uint32_t>(bitcast_u32(a.x), bitcast_u32(a.y), bitcast_u32(a.z)); }
template <class S> ND_HD_INLINE v4<uint32_t> vbitcast_u32(v4<S> a) { return v4<uint32_t>(bitcast_u32(a.x), bitcast_u32(a.y), bitcast_u32(a.z), bitcast_u32(a.w)); }

// component-wise float builtins on vectors
#define ND_VFUN1(NAME)                                                               \
  template <class S> ND_HD_INLINE v2<S> NAME(v2<S> a) { return v2<S>(NAME(a.x), NAME(a.y)); } \
  template <class S> ND_HD_INLINE v3<S> NAME(v3<S> a) { return v3<S>(NAME(a.x), NAME(a.y), NAME(a.z)); } \
  template <class S> ND_HD_INLINE v4<S> NAME(v4<S> a) { return v4<S>(NAME(a.x), NAME(a.y), NAME(a.z), NAME(a.w)); }
ND_VFUN1(sin) ND_VFUN1(cos) ND_VFUN1(tan) ND_VFUN1(asin) ND_VFUN1(acos) ND_VFUN1(atan)
ND_VFUN1(sinh) ND_VFUN1(cosh) ND_VFUN1(tanh)
ND_VFUN1(exp) ND_VFUN1(exp2) ND_VFUN1(log) ND_VFUN1(log2) ND_VFUN1(sqrt) ND_VFUN1(inverseSqrt)
ND_VFUN1(floor) ND_VFUN1(ceil) ND_VFUN1(trunc) ND_VFUN1(round) ND_VFUN1(fract)
ND_VFUN1(radians) ND_VFUN1(degrees) ND_VFUN1(abs) ND_VFUN1(sign) ND_VFUN1(saturate)
#undef ND_VFUN1

#define ND_VFUN2(NAME)                                                                          \
  template <class S> ND_HD_INLINE v2<S> NAME(v2<S> a, v2<S> b) { return v2<S>(NAME(a.x, b.x), NAME(a.y, b.y)); } \
  template <class S> ND_HD_INLINE v3<S> NAME(v3<S> a, v3<S> b) { return v3<S>(NAME(a.x, b.x), NAME(a.y, b.y), NAME(a.z, b.z)); } \
  template <class S> ND_HD_INLINE v4<S> NAME(v4<S> a, v4<S> b) { return v4<S>(NAME(a.x, b.x), NAME(a.y, b.y), NAME(a.z, b.z), NAME(a.w, b.w)); }
ND_VFUN2(min) ND_VFUN2(max) ND_VFUN2(pow) ND_VFUN2(atan2) ND_VFUN2(step) ND_VFUN2(fmod_trunc)
#undef ND_VFUN2

template <class S> ND_HD_INLINE v2<S> clamp(v2<S> x, v2<S> lo, v2<S> hi) { return min(max(x, lo), hi); }
template <class S> ND_HD_INLINE v3<S> clamp(v3<S> x, v3<S> lo, v3<S> hi) { return min(max(x, lo), hi); }
template <class S> ND_HD_INLINE v4<S> clamp(v4<S> x, v4<S> lo, v4<S> hi) { return min(max(x, lo), hi); }
template <class S> ND_HD_INLINE v2<S> mix(v2<S> a, v2<S> b, v2<S> t) { return a * (v2<S>(S(1)) - t) + b * t; }
template <class S> ND_HD_INLINE v3<S> mix(v3<S> a, v3<S> b, v3<S> t) { return a * (v3<S>(S(1)) - t) + b * t; }
template <class S> ND_HD_INLINE v4<S> mix(v4<S> a, v4<S> b, v4<S> t) { return a * (v4<S>(S(1)) - t) + b * t; }
template <class S> ND_HD_INLINE v2<S> mix(v2<S> a, v2<S> b, S t) { return a * (S(1) - t) + b * t; }
template <class S> ND_HD_INLINE v3<S> mix(v3<S> a, v3<S> b, S t) { return a * (S(1) - t) + b * t; }
template <class S> ND_HD_INLINE v4<S> mix(v4<S> a, v4<S> b, S t) { return a * (S(1) - t) + b * t; }
#define ND_VFUN3(NAME)                                                                          \
  template <class S> ND_HD_INLINE v2<S> NAME(v2<S> a, v2<S> b, v2<S> c) { return v2<S>(NAME(a.x, b.x, c.x), NAME(a.y, b.y, c.y)); } \
  template <class S> ND_HD_INLINE v3<S> NAME(v3<S> a, v3<S> b, v3<S> c) { return v3<S>(NAME(a.x, b.x, c.x), NAME(a.y, b.y, c.y), NAME(a.z, b.z, c.z)); } \
  template <class S> ND_HD_INLINE v4<S> NAME(v4<S> a, v4<S> b, v4<S> c) { return v4<S>(NAME(a.x, b.x, c.x), NAME(a.y, b.y, c.y), NAME(a.z, b.z, c.z), NAME(a.w, b.w, c.w)); }
ND_VFUN3(smoothstep) ND_VFUN3(fma)
#undef ND_VFUN3

template <class S> ND_HD_INLINE v2<S> select(v2<S> f, v2<S> t, bool c) { return c ? t : f; }
template <class S> ND_HD_INLINE v3<S> select(v3<S> f, v3<S> t, bool c) { return c ? t : f; }
template <class S> ND_HD_INLINE v4<S> select(v4<S> f, v4<S> t, bool c) { return c ? t : f; }
template <class S> ND_HD_INLINE v2<S> select(v2<S> f, v2<S> t, v2<bool> c) { return v2<S>(c.x ? t.x : f.x, c.y ? t.y : f.y); }
template <class S> ND_HD_INLINE v3<S> select(v3<S> f, v3<S> t, v3<bool> c) { return v3<S>(c.x ? t.x : f.x, c.y ? t.y : f.y, c.z ? t.z : f.z); }
template <class S> ND_HD_INLINE v4<S> select(v4<S> f, v4<S> t, v4<bool> c) { return v4<S>(c.x ? t.x : f.x, c.y ? t.y : f.y, c.z ? t.z : f.z, c.w ? t.w : f.w); }

// The scalar type of a value (a vector's component type).
template <class X> struct scalar_of { typedef X type; };
template <class S> struct scalar_of<v2<S>> { typedef S type; };
template <class S> struct scalar_of<v3<S>> { typedef S type; };
template <class S> struct scalar_of<v4<S>> { typedef S type; };

// (a + b) + c where b and c are the same in every iteration of a formula's de_step
// (built from pos and the parameters only).  The FP32 DE on the device adds b + c
// first, so that the compiler computes it once per DE evaluation, outside the
// iteration loop; the one rounding of that sum moves.  The FP64 DE, the dual numbers
// and host code keep WGSL's left-to-right order.
template <class A, class B, class C>
ND_HD_INLINE auto add_inv(const A& a, const B& b, const C& c) -> decltype((a + b) + c) {
#if defined(__CUDA_ARCH__) && !defined(ND_OPCOUNT_BUILD)
  if constexpr (std::is_same<typename scalar_of<A>::type, float>::value) return a + (b + c);
#endif
  return (a + b) + c;
}

template <class S> ND_HD_INLINE S dot(v2<S> a, v2<S> b) { return a.x * b.x + a.y * b.y; }
template <class S> ND_HD_INLINE S dot(v3<S> a, v3<S> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S> ND_HD_INLINE S dot(v4<S> a, v4<S> b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
template <class V> ND_HD_INLINE auto length(V a) { return sqrt(dot(a, a)); }
template <class V> ND_HD_INLINE auto distance(V a, V b) { return length(a - b); }
template <class V> ND_HD_INLINE V normalize(V a) {
  auto inv = decltype(a.x)(1) / length(a);
  return a * inv;
}
template <class S> ND_HD_INLINE v3<S> cross(v3<S> a, v3<S> b) {
  return v3<S>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class V> ND_HD_INLINE V reflect(V e1, V e2) { return e1 - e2 * (decltype(e1.x)(2) * dot(e2, e1)); }

// ---------------------------------------------------------------- matrices (column-major)
template <class T> struct m2 {
  v2<T> c[2];
  ND_HD_INLINE m2() {}
  ND_HD_INLINE m2(v2<T> a, v2<T> b) { c[0] = a; c[1] = b; }
  ND_HD_INLINE v2<T>& operator[](int i) { return c[i <= 0 ? 0 : 1]; }
  ND_HD_INLINE v2<T> operator[](int i) const { return c[i <= 0 ? 0 : 1]; }
  ND_HD_INLINE v2<T>& operator[](uint32_t i) { return c[i >= 1u ? 1 : 0]; }
  ND_HD_INLINE v2<T> operator[](uint32_t i) const { return c[i >= 1u ? 1 : 0]; }
};
template <class T> struct m3 {
  v3<T> c[3];
  ND_HD_INLINE m3() {}
  ND_HD_INLINE m3(v3<T> a, v3<T> b, v3<T> d) { c[0] = a; c[1] = b; c[2] = d; }
  ND_HD_INLINE v3<T>& operator[](int i) { return c[i <= 0 ? 0 : (i >= 2 ? 2 : i)]; }
  ND_HD_INLINE v3<T> operator[](int i) const { return c[i <= 0 ? 0 : (i >= 2 ? 2 : i)]; }
  ND_HD_INLINE v3<T>& operator[](uint32_t i) { return c[i >= 2u ? 2 : int(i)]; }
  ND_HD_INLINE v3<T> operator[](uint32_t i) const { return c[i >= 2u ? 2 : int(i)]; }
};
template <class T> struct m4 {
  v4<T> c[4];
  ND_HD_INLINE m4() {}
  ND_HD_INLINE m4(v4<T> a, v4<T> b, v4<T> d, v4<T> e) { c[0] = a; c[1] = b; c[2] = d; c[3] = e; }
  ND_HD_INLINE v4<T>& operator[](int i) { return c[i <= 0 ? 0 : (i >= 3 ? 3 : i)]; }
  ND_HD_INLINE v4<T> operator[](int i) const { return c[i <= 0 ? 0 : (i >= 3 ? 3 : i)]; }
};

template <class T> ND_HD_INLINE v2<T> mul(m2<T> m, v2<T> v) { return m.c[0] * v.x + m.c[1] * v.y; }
template <class T> ND_HD_INLINE v3<T> mul(m3<T> m, v3<T> v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z; }
template <class T> ND_HD_INLINE v4<T> mul(m4<T> m, v4<T> v) { return m.c[0] * v.x + m.c[1] * v.y + m.c[2] * v.z + m.c[3] * v.w; }
template <class T> ND_HD_INLINE v2<T> mul(v2<T> v, m2<T> m) { return v2<T>(dot(v, m.c[0]), dot(v, m.c[1])); }
template <class T> ND_HD_INLINE v3<T> mul(v3<T> v, m3<T> m) { return v3<T>(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2])); }
template <class T> ND_HD_INLINE v4<T> mul(v4<T> v, m4<T> m) { return v4<T>(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2]), dot(v, m.c[3])); }
template <class T> ND_HD_INLINE m2<T> mul(m2<T> a, m2<T> b) { return m2<T>(mul(a, b.c[0]), mul(a, b.c[1])); }
template <class T> ND_HD_INLINE m3<T> mul(m3<T> a, m3<T> b) { return m3<T>(mul(a, b.c[0]), mul(a, b.c[1]), mul(a, b.c[2])); }
template <class T> ND_HD_INLINE m4<T> mul(m4<T> a, m4<T> b) { return m4<T>(mul(a, b.c[0]), mul(a, b.c[1]), mul(a, b.c[2]), mul(a, b.c[3])); }
template <class T> ND_HD_INLINE m2<T> operator*(m2<T> a, T s) { return m2<T>(a.c[0] * s, a.c[1] * s); }
template <class T> ND_HD_INLINE m3<T> operator*(m3<T> a, T s) { return m3<T>(a.c[0] * s, a.c[1] * s, a.c[2] * s); }
template <class T> ND_HD_INLINE m2<T> operator+(m2<T> a, m2<T> b) { return m2<T>(a.c[0] + b.c[0], a.c[1] + b.c[1]); }
template <class T> ND_HD_INLINE m3<T> operator+(m3<T> a, m3<T> b) { return m3<T>(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]); }
template <class T> ND_HD_INLINE m2<T> operator-(m2<T> a, m2<T> b) { return m2<T>(a.c[0] - b.c[0], a.c[1] - b.c[1]); }
template <class T> ND_HD_INLINE m3<T> operator-(m3<T> a, m3<T> b) { return m3<T>(a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]); }
template <class T> ND_HD_INLINE m3<T> operator-(m3<T> a) { return m3<T>(-a.c[0], -a.c[1], -a.c[2]); }
template <class T> ND_HD_INLINE m2<T> transpose(m2<T> m) {
  return m2<T>(v2<T>(m.c[0].x, m.c[1].x), v2<T>(m.c[0].y, m.c[1].y));
}
template <class T> ND_HD_INLINE m3<T> transpose(m3<T> m) {
  return m3<T>(v3<T>(m.c[0].x, m.c[1].x, m.c[2].x), v3<T>(m.c[0].y, m.c[1].y, m.c[2].y),
               v3<T>(m.c[0].z, m.c[1].z, m.c[2].z));
}
template <class T> ND_HD_INLINE T determinant(m2<T> m) { return m.c[0].x * m.c[1].y - m.c[1].x * m.c[0].y; }
template <class T> ND_HD_INLINE T determinant(m3<T> m) { return dot(m.c[0], cross(m.c[1], m.c[2])); }

// ---------------------------------------------------------------- fixed arrays
template <class E, int N> struct arr {
  E v[N];
  ND_HD_INLINE E& operator[](int i) { return v[i < 0 ? 0 : (i >= N ? N - 1 : i)]; }
  ND_HD_INLINE const E& operator[](int i) const { return v[i < 0 ? 0 : (i >= N ? N - 1 : i)]; }
  ND_HD_INLINE E& operator[](uint32_t i) { return v[i >= uint32_t(N) ? N - 1 : int(i)]; }
  ND_HD_INLINE const E& operator[](uint32_t i) const { return v[i >= uint32_t(N) ? N - 1 : int(i)]; }
};

// ---------------------------------------------------------------- formula state
// The state a formula's de_step receives and returns (template.wgsl:97-100).
template <class T> struct IterCarry {
  v3<T> z;
  T dr;
};

// Params access: p[i] with i clamped to the 16 slots (template.wgsl:102-104).
template <class P> ND_HD_INLINE auto param(const P& p, int i) { return p[i < 0 ? 0 : (i > 15 ? 15 : i)]; }
template <class P> ND_HD_INLINE auto param(const P& p, uint32_t i) { return p[i > 15u ? 15 : int(i)]; }

#undef ND_MAP1

}  // namespace ndw
