// Op-counting float type for the host build of the ray program (nd_opcount.cpp).
//
// The algorithmic FLOP count of a launch is the sum, over its DE evaluations, of
// the floating-point operations the formula code performs.  Running the very same
// formula and march code with T = CF on the host counts them exactly:
//   flops = add + mul + div + 2 * fma   (one FP32 add/sub/mul/div = 1 FLOP)
//   sfu   = transcendental and square-root calls (sin, cos, acos, atan2, pow, log,
//           exp, sqrt, ...), reported beside the FLOPs
//   other = compares, min/max/abs/floor/round/select and conversions
#pragma once

#include <math.h>
#include <stdint.h>

namespace ndw {

struct OpCounts {
  uint64_t add = 0, mul = 0, div = 0, fma = 0, sfu = 0, other = 0;
  uint64_t flops() const { return add + mul + div + 2 * fma; }
};

inline OpCounts& op_counts() {
  static thread_local OpCounts c;
  return c;
}

struct CF {
  float v;
  CF() : v(0.0f) {}
  CF(float x) : v(x) {}
  CF(double x) : v(float(x)) {}
  CF(int x) : v(float(x)) {}
  CF(unsigned x) : v(float(x)) {}
  CF(long x) : v(float(x)) {}
  explicit operator float() const { return v; }
  explicit operator double() const { return double(v); }
  CF& operator+=(CF o) { ++op_counts().add; v += o.v; return *this; }
  CF& operator-=(CF o) { ++op_counts().add; v -= o.v; return *this; }
  CF& operator*=(CF o) { ++op_counts().mul; v *= o.v; return *this; }
  CF& operator/=(CF o) { ++op_counts().div; v /= o.v; return *this; }
};

inline CF operator+(CF a, CF b) { ++op_counts().add; return CF(a.v + b.v); }
inline CF operator-(CF a, CF b) { ++op_counts().add; return CF(a.v - b.v); }
inline CF operator*(CF a, CF b) { ++op_counts().mul; return CF(a.v * b.v); }
inline CF operator/(CF a, CF b) { ++op_counts().div; return CF(a.v / b.v); }
inline CF operator-(CF a) { return CF(-a.v); }
#define ND_CF_CMP(OP) \
  inline bool operator OP(CF a, CF b) { ++op_counts().other; return a.v OP b.v; }
ND_CF_CMP(<) ND_CF_CMP(>) ND_CF_CMP(<=) ND_CF_CMP(>=) ND_CF_CMP(==) ND_CF_CMP(!=)
#undef ND_CF_CMP

#define ND_CF_SFU1(NAME, F) \
  inline CF NAME(CF x) { ++op_counts().sfu; return CF(F(x.v)); }
ND_CF_SFU1(sin, sinf) ND_CF_SFU1(cos, cosf) ND_CF_SFU1(tan, tanf) ND_CF_SFU1(asin, asinf)
ND_CF_SFU1(acos, acosf) ND_CF_SFU1(atan, atanf) ND_CF_SFU1(sinh, sinhf) ND_CF_SFU1(cosh, coshf)
ND_CF_SFU1(tanh, tanhf) ND_CF_SFU1(exp, expf) ND_CF_SFU1(exp2, exp2f) ND_CF_SFU1(log, logf)
ND_CF_SFU1(log2, log2f) ND_CF_SFU1(sqrt, sqrtf)
#undef ND_CF_SFU1
inline CF inverseSqrt(CF x) { ++op_counts().sfu; return CF(1.0f / sqrtf(x.v)); }
inline CF pow(CF x, CF y) { ++op_counts().sfu; return CF(x.v < 0.0f ? __builtin_nanf("") : powf(x.v, y.v)); }
inline CF atan2(CF y, CF x) { ++op_counts().sfu; return CF(atan2f(y.v, x.v)); }

#define ND_CF_OTHER1(NAME, EXPR) \
  inline CF NAME(CF a) { ++op_counts().other; const float x = a.v; return CF(EXPR); }
ND_CF_OTHER1(floor, floorf(x)) ND_CF_OTHER1(ceil, ceilf(x)) ND_CF_OTHER1(trunc, truncf(x))
ND_CF_OTHER1(round, rintf(x)) ND_CF_OTHER1(abs, fabsf(x))
ND_CF_OTHER1(sign, x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f))
#undef ND_CF_OTHER1
inline CF radians(CF x) { ++op_counts().mul; return CF(x.v * 0.017453292519943295f); }
inline CF degrees(CF x) { ++op_counts().mul; return CF(x.v * 57.29577951308232f); }
inline CF min(CF a, CF b) { ++op_counts().other; return CF(fminf(a.v, b.v)); }
inline CF max(CF a, CF b) { ++op_counts().other; return CF(fmaxf(a.v, b.v)); }
inline CF fma(CF a, CF b, CF c) { ++op_counts().fma; return CF(fmaf(a.v, b.v, c.v)); }
inline CF select(CF f, CF t, bool c) { ++op_counts().other; return c ? t : f; }

}  // namespace ndw

#include "nd_rayprog.h"

namespace nd {

// Runs the ray program of one ray on the host with T = CF and adds the ops of all
// its DE evaluations to *out (the program's own bookkeeping runs in double and is
// not counted).
template <class Set>
inline void count_ray(const DevView& view, int64_t ray, ndw::OpCounts* out, uint32_t* evals) {
  DevView v = view;
  v.out_offset = -(ray - v.ray_offset);  // write this ray's outputs to slot 0
  float depth = 0.0f;
  nd_gbuffer g;
  memset(&g, 0, sizeof(g));
  g.depth = &depth;
  ndw::OpCounts& c = ndw::op_counts();
  const ndw::OpCounts before = c;
  Lane<ndw::CF, false> L;
  L.start(v, int32_t(ray), 0);
  if (L.phase == PH_DONE) L.finish(v, g, nullptr, 1.0f);
  while (L.phase != PH_DONE) {
    const DEOut<ndw::CF> de = Set::template de<ndw::CF>(v.code, to_t<ndw::CF>(L.sample_pos(v)), v);
    L.advance(v, de, g, nullptr);
  }
  if (L.hit) {  // the trap pass: one DE with the orbit trap at the hit point
    ++*evals;
    g.trap = &depth;
    trap_at_hit<Set, ndw::CF, false>(v, ray - v.ray_offset, L.t, g, nullptr);
  }
  out->add += c.add - before.add;
  out->mul += c.mul - before.mul;
  out->div += c.div - before.div;
  out->fma += c.fma - before.fma;
  out->sfu += c.sfu - before.sfu;
  out->other += c.other - before.other;
  *evals += L.evals;
}

}  // namespace nd
