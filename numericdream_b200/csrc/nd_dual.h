// Forward-mode dual numbers (value + one tangent) for the adjoint pass.
//
// Instantiating the translated formula code with T = Dual<S> carries the
// directional derivative of every intermediate along one tangent: seeding the
// position with dp/dtheta and the parameters with dparams/dtheta yields dDE/dtheta in
// one evaluation.  Functions follow their derivative rules; piecewise-constant ones
// (floor, round, sign, comparisons) have a zero tangent, and min/max/select follow
// the branch the value takes.  S is float (Dual1, the FP32 adjoint) or double.
#pragma once

#include "nd_wgsl.h"

namespace ndw {

template <class S> struct Dual {
  S v, d;
  ND_HD_INLINE Dual() : v(S(0)), d(S(0)) {}
  ND_HD_INLINE Dual(float x) : v(S(x)), d(S(0)) {}
  ND_HD_INLINE Dual(double x) : v(S(x)), d(S(0)) {}
  ND_HD_INLINE Dual(int x) : v(S(x)), d(S(0)) {}
  ND_HD_INLINE Dual(unsigned x) : v(S(x)), d(S(0)) {}
  ND_HD_INLINE Dual(S x, S t, int) : v(x), d(t) {}
  ND_HD_INLINE explicit operator float() const { return float(v); }
  ND_HD_INLINE explicit operator double() const { return double(v); }
  ND_HD_INLINE Dual& operator+=(Dual o) { v += o.v; d += o.d; return *this; }
  ND_HD_INLINE Dual& operator-=(Dual o) { v -= o.v; d -= o.d; return *this; }
  ND_HD_INLINE Dual& operator*=(Dual o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
  ND_HD_INLINE Dual& operator/=(Dual o) {
    const S q = v / o.v;
    d = (d - q * o.d) / o.v;
    v = q;
    return *this;
  }
};
typedef Dual<float> Dual1;

template <class S> ND_HD_INLINE Dual<S> mkd(S v, S d) { return Dual<S>(v, d, 0); }

template <class S> ND_HD_INLINE Dual<S> operator+(Dual<S> a, Dual<S> b) { return mkd(a.v + b.v, a.d + b.d); }
template <class S> ND_HD_INLINE Dual<S> operator-(Dual<S> a, Dual<S> b) { return mkd(a.v - b.v, a.d - b.d); }
template <class S> ND_HD_INLINE Dual<S> operator*(Dual<S> a, Dual<S> b) { return mkd(a.v * b.v, a.d * b.v + a.v * b.d); }
template <class S> ND_HD_INLINE Dual<S> operator/(Dual<S> a, Dual<S> b) {
  const S q = a.v / b.v;
  return mkd(q, (a.d - q * b.d) / b.v);
}
template <class S> ND_HD_INLINE Dual<S> operator-(Dual<S> a) { return mkd(-a.v, -a.d); }
template <class S> ND_HD_INLINE bool operator<(Dual<S> a, Dual<S> b) { return a.v < b.v; }
template <class S> ND_HD_INLINE bool operator>(Dual<S> a, Dual<S> b) { return a.v > b.v; }
template <class S> ND_HD_INLINE bool operator<=(Dual<S> a, Dual<S> b) { return a.v <= b.v; }
template <class S> ND_HD_INLINE bool operator>=(Dual<S> a, Dual<S> b) { return a.v >= b.v; }
template <class S> ND_HD_INLINE bool operator==(Dual<S> a, Dual<S> b) { return a.v == b.v; }
template <class S> ND_HD_INLINE bool operator!=(Dual<S> a, Dual<S> b) { return a.v != b.v; }

template <class S> ND_HD_INLINE Dual<S> sin(Dual<S> a) { return mkd(sin(a.v), cos(a.v) * a.d); }
template <class S> ND_HD_INLINE Dual<S> cos(Dual<S> a) { return mkd(cos(a.v), -sin(a.v) * a.d); }
template <class S> ND_HD_INLINE Dual<S> tan(Dual<S> a) {
  const S t = tan(a.v);
  return mkd(t, (S(1) + t * t) * a.d);
}
template <class S> ND_HD_INLINE Dual<S> asin(Dual<S> a) {
  return mkd(asin(a.v), a.d / sqrt(max(S(1) - a.v * a.v, S(1e-30))));
}
template <class S> ND_HD_INLINE Dual<S> acos(Dual<S> a) {
  return mkd(acos(a.v), -a.d / sqrt(max(S(1) - a.v * a.v, S(1e-30))));
}
template <class S> ND_HD_INLINE Dual<S> atan(Dual<S> a) { return mkd(atan(a.v), a.d / (S(1) + a.v * a.v)); }
template <class S> ND_HD_INLINE Dual<S> atan2(Dual<S> y, Dual<S> x) {
  const S r2 = x.v * x.v + y.v * y.v;
  return mkd(atan2(y.v, x.v), r2 > S(0) ? (x.v * y.d - y.v * x.d) / r2 : S(0));
}
template <class S> ND_HD_INLINE Dual<S> sinh(Dual<S> a) { return mkd(sinh(a.v), cosh(a.v) * a.d); }
template <class S> ND_HD_INLINE Dual<S> cosh(Dual<S> a) { return mkd(cosh(a.v), sinh(a.v) * a.d); }
template <class S> ND_HD_INLINE Dual<S> tanh(Dual<S> a) {
  const S t = tanh(a.v);
  return mkd(t, (S(1) - t * t) * a.d);
}
template <class S> ND_HD_INLINE Dual<S> exp(Dual<S> a) {
  const S e = exp(a.v);
  return mkd(e, e * a.d);
}
template <class S> ND_HD_INLINE Dual<S> exp2(Dual<S> a) {
  const S e = exp2(a.v);
  return mkd(e, e * S(0.6931471805599453) * a.d);
}
template <class S> ND_HD_INLINE Dual<S> log(Dual<S> a) { return mkd(log(a.v), a.d / a.v); }
template <class S> ND_HD_INLINE Dual<S> log2(Dual<S> a) { return mkd(log2(a.v), a.d / (a.v * S(0.6931471805599453))); }
template <class S> ND_HD_INLINE Dual<S> sqrt(Dual<S> a) {
  const S s = sqrt(a.v);
  return mkd(s, s > S(0) ? a.d / (S(2) * s) : S(0));
}
template <class S> ND_HD_INLINE Dual<S> inverseSqrt(Dual<S> a) {
  const S r = S(1) / sqrt(a.v);
  return mkd(r, S(-0.5) * r * r * r * a.d);
}
template <class S> ND_HD_INLINE Dual<S> pow(Dual<S> x, Dual<S> y) {
  if (x.v < S(0)) return mkd(S(0) / S(0), S(0));
  const S p = pow(x.v, y.v);
  S dp = S(0);
  if (x.d != S(0)) dp += y.v * pow(x.v, y.v - S(1)) * x.d;
  if (y.d != S(0) && x.v > S(0)) dp += p * log(x.v) * y.d;
  return mkd(p, dp);
}
template <class S> ND_HD_INLINE Dual<S> floor(Dual<S> a) { return mkd(floor(a.v), S(0)); }
template <class S> ND_HD_INLINE Dual<S> ceil(Dual<S> a) { return mkd(ceil(a.v), S(0)); }
template <class S> ND_HD_INLINE Dual<S> trunc(Dual<S> a) { return mkd(trunc(a.v), S(0)); }
template <class S> ND_HD_INLINE Dual<S> round(Dual<S> a) { return mkd(round(a.v), S(0)); }
template <class S> ND_HD_INLINE Dual<S> abs(Dual<S> a) { return a.v < S(0) ? -a : a; }
template <class S> ND_HD_INLINE Dual<S> sign(Dual<S> a) {
  return mkd(a.v > S(0) ? S(1) : (a.v < S(0) ? S(-1) : S(0)), S(0));
}
template <class S> ND_HD_INLINE Dual<S> min(Dual<S> a, Dual<S> b) { return b.v < a.v ? b : a; }
template <class S> ND_HD_INLINE Dual<S> max(Dual<S> a, Dual<S> b) { return b.v > a.v ? b : a; }
template <class S> ND_HD_INLINE Dual<S> fma(Dual<S> a, Dual<S> b, Dual<S> c) { return a * b + c; }
template <class S> ND_HD_INLINE Dual<S> radians(Dual<S> a) {
  return mkd(a.v * S(0.017453292519943295), a.d * S(0.017453292519943295));
}
template <class S> ND_HD_INLINE Dual<S> degrees(Dual<S> a) {
  return mkd(a.v * S(57.29577951308232), a.d * S(57.29577951308232));
}
template <class S> ND_HD_INLINE Dual<S> select(Dual<S> f, Dual<S> t, bool c) { return c ? t : f; }
template <class S> ND_HD_INLINE void sin_cos(Dual<S> x, Dual<S>& s, Dual<S>& c) {
  const S sv = sin(x.v), cv = cos(x.v);
  s = mkd(sv, cv * x.d);
  c = mkd(cv, -sv * x.d);
}

}  // namespace ndw
