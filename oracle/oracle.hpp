// CPU oracle for the distance-estimator sphere-tracing pass.  TEST INFRASTRUCTURE:
// only tests, the smoke check and bench.py's CPU-baseline leg use this code, as the
// checker and the timed CPU baseline; the CUDA product never calls it.
//
// This is an independent, hand-written restatement of NumericDream's WGSL (the
// reference app's src/gpu/shaders/template.wgsl, "tpl" below, and the formula
// files), templated on the float type R: R = double is the FP64 oracle every error
// figure is measured against, R = float mirrors the reference's own f32 arithmetic
// and is the timed CPU baseline.  It shares no code with the CUDA library.
//
// Parity pinning: the reference ships no golden vectors, known-answer tests or
// fixtures for this path, and it cannot run here (Zig, wgpu-native and a graphics
// stack are all absent).  The formulas below are pinned instead (a) against the
// reference's own formula sources, mechanically translated and compiled under
// oracle/_ref (see build_ref.py), on fixed point sets committed as tests/golden
// fixtures, and (b) against closed-form answers for the sphere and cube
// primitives.  The march (march_to with its bisection, verify and high-quality
// modes, march_epsilon) and the tetrahedral normal are pinned the same way as (a):
// the reference's own functions of the shader template, translated mechanically and
// compiled under oracle/_ref, traced the same rays in FP64, and this restatement
// matches the committed results bit for bit (hit, t, steps, evaluations); so are
// the orbit trap (the reference's generated formula wrapper and trap functions) and
// the combine modes (its combine_de), the opaque shadow ray (visibility_march) and
// the Lambert level (simple_geometry).  The central-difference normal, the scene
// assembly and the accelerator are pinned by closed forms and reading only.
#pragma once

#include <stdint.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <string>
#include <vector>

#include "../include/nd_march.h"

namespace oracle {

template <class R> struct V3 {
  R x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(R a, R b, R c) : x(a), y(b), z(c) {}
  explicit V3(R s) : x(s), y(s), z(s) {}
  V3 operator+(V3 o) const { return V3(x + o.x, y + o.y, z + o.z); }
  V3 operator-(V3 o) const { return V3(x - o.x, y - o.y, z - o.z); }
  V3 operator*(R s) const { return V3(x * s, y * s, z * s); }
  V3 operator/(R s) const { return V3(x / s, y / s, z / s); }
  V3 operator-() const { return V3(-x, -y, -z); }
};
template <class R> R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> R len(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> V3<R> norm(V3<R> a) { return a * (R(1) / len(a)); }
template <class R> V3<R> vabs(V3<R> a) { return V3<R>(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
template <class R> V3<R> vmax(V3<R> a, R s) { return V3<R>(std::fmax(a.x, s), std::fmax(a.y, s), std::fmax(a.z, s)); }
template <class R> V3<R> cross(V3<R> a, V3<R> b) {
  return V3<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class R> R clampv(R x, R lo, R hi) { return std::fmin(std::fmax(x, lo), hi); }

template <class R> struct Carry {
  V3<R> z;
  R dr;
};

// ------------------------------------------------------------------ formulas
// Each formula: iterations(p), step(carry, pos, p), finalize(carry).

// Built-in Mandelbulb: src/gpu/shaders/mandelbrot.wgsl:1-13 with bulb_power_step
// (tpl:1019-1031, BULB_BAILOUT = 2 tpl:1013) and bulb_log_escape (tpl:1006-1010).
template <class R> struct Mandelbulb {
  static int iterations(const R* p) { return to_int(p[1]); }
  static Carry<R> step(Carry<R> c, V3<R> pos, const R* p) {
    const R power = p[0];
    const R r = len(c.z);
    if (r > R(2)) return c;
    const R theta = std::acos(clampv(c.z.z / r, R(-1), R(1))) * power;
    const R phi = std::atan2(c.z.y, c.z.x) * power;
    const R rp = std::pow(r, power - R(1));
    Carry<R> o;
    o.dr = rp * power * c.dr + R(1);
    const R zr = rp * r;
    o.z = V3<R>(std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi), std::cos(theta)) * zr + pos;
    return o;
  }
  static R finalize(Carry<R> c) {
    const R r = len(c.z);
    const R est = R(0.5) * std::log(std::fmax(r, R(1e-6))) * r / std::fmax(c.dr, R(1e-6));
    return std::fmin(est, r);
  }
  static int to_int(R v) { return int(v); }
};

// Euler rotation in degrees about x, then y, then z (rotate_xyz_deg tpl:1085-1093,
// rot_x/rot_y/rot_z tpl:1392-1408); identity when all angles are zero.
template <class R> V3<R> rotate_deg(V3<R> z, R ax, R ay, R az) {
  if (ax == R(0) && ay == R(0) && az == R(0)) return z;
  const R k = R(0.017453292519943295);
  R a = ax * k, b = ay * k, g = az * k;
  // rot_x(a) * z
  R c = std::cos(a), s = std::sin(a);
  V3<R> v(z.x, c * z.y - s * z.z, s * z.y + c * z.z);
  // rot_y(b) * v
  c = std::cos(b); s = std::sin(b);
  v = V3<R>(c * v.x + s * v.z, v.y, -s * v.x + c * v.z);
  // rot_z(g) * v
  c = std::cos(g); s = std::sin(g);
  return V3<R>(c * v.x - s * v.y, s * v.x + c * v.y, v.z);
}

// Mandelbox: formulas/amazingbox_box.wgsl:13-36 with box_fold (tpl:949),
// sphere_fold (tpl:959), de_finalize_scaled (tpl:993).
template <class R> struct Mandelbox {
  static int iterations(const R* p) { return int(p[4]); }
  static Carry<R> step(Carry<R> c, V3<R> pos, const R* p) {
    const R scale = p[0];
    const R min_r2 = p[1] * p[1];
    const R fixed_r2 = p[2] * p[2];
    const R lim = p[3];
    V3<R> z(clampv(c.z.x, -lim, lim) * R(2) - c.z.x, clampv(c.z.y, -lim, lim) * R(2) - c.z.y,
            clampv(c.z.z, -lim, lim) * R(2) - c.z.z);
    R dr = c.dr;
    const R r2 = dot(z, z);
    if (r2 < min_r2) {
      const R t = fixed_r2 / min_r2;
      z = z * t;
      dr = dr * t;
    } else if (r2 < fixed_r2) {
      const R t = fixed_r2 / r2;
      z = z * t;
      dr = dr * t;
    }
    z = rotate_deg(z, p[5], p[6], p[7]);
    z = z * scale + pos * p[8] + V3<R>(p[9], p[10], p[11]);
    dr = dr * std::fabs(scale) + std::fmax(std::fabs(p[8]), R(1));
    return Carry<R>{z, dr};
  }
  static R finalize(Carry<R> c) { return len(c.z) / std::fabs(c.dr); }
};

// Menger sponge: formulas/menger3_ifs.wgsl:9-28 with sort_desc_abs (tpl:1036).
template <class R> struct Menger3 {
  static int iterations(const R* p) { return int(p[0]); }
  static Carry<R> step(Carry<R> c, V3<R>, const R* p) {
    const R scale = p[4];
    const V3<R> off(p[1], p[2], p[3]);
    V3<R> v = vabs(c.z);
    if (v.x < v.y) std::swap(v.x, v.y);
    if (v.x < v.z) std::swap(v.x, v.z);
    if (v.y < v.z) std::swap(v.y, v.z);
    V3<R> z = rotate_deg(v, p[5], p[6], p[7]);
    z = z * scale - off * (scale - R(1));
    if (z.z < R(-0.5) * off.z * (scale - R(1))) z.z = z.z + off.z * (scale - R(1));
    return Carry<R>{z, c.dr * scale};
  }
  static R finalize(Carry<R> c) {
    const V3<R> q = vabs(c.z) - V3<R>(R(1));
    return len(vmax(q, R(0))) / c.dr;
  }
};

// Pseudo-Kleinian: formulas/pseudokleinian_kleinian.wgsl:11-33 with lattice_wrap
// (tpl:987, round half to even) and sphere_invert_offset (tpl:975).
template <class R> struct PseudoKleinian {
  static int iterations(const R* p) { return int(p[5]); }
  static R rne(R x) { return std::nearbyint(x); }
  static Carry<R> step(Carry<R> c, V3<R> pos, const R* p) {
    const V3<R> center(p[0], p[1], p[2]);
    const R radius2 = p[3] * p[3];
    const R cell = p[4];
    V3<R> z(c.z.x - cell * rne(c.z.x / cell), c.z.y - cell * rne(c.z.y / cell), c.z.z - cell * rne(c.z.z / cell));
    R dr = c.dr;
    const V3<R> d = z - center;
    const R r2 = std::fmax(dot(d, d), R(1e-6));
    if (r2 < radius2) {
      const R t = radius2 / r2;
      z = center + d * t;
      dr = dr * t;
    }
    z = z + pos * p[6] + V3<R>(p[7], p[8], p[9]);
    dr = dr + std::fmax(std::fabs(p[6]), R(1));
    return Carry<R>{z, dr};
  }
  static R finalize(Carry<R> c) { return len(c.z) / std::fabs(c.dr); }
};

// Primitives: formulas/sphere_primitive.wgsl, formulas/cube_primitive.wgsl with
// primitive_de_step (tpl:1100-1109).
template <class R> Carry<R> primitive_step(Carry<R> c, R size) {
  const R unit = R(1) / std::fmax(size, R(1e-4));
  const R f = unit / std::fmax(std::fabs(c.dr), R(1e-6));
  return Carry<R>{c.z * f, unit};
}
template <class R> struct SpherePrim {
  static int iterations(const R*) { return 1; }
  static Carry<R> step(Carry<R> c, V3<R>, const R* p) { return primitive_step(c, p[0]); }
  static R finalize(Carry<R> c) { return (len(c.z) - R(1)) / std::fmax(std::fabs(c.dr), R(1e-6)); }
};
template <class R> struct CubePrim {
  static int iterations(const R*) { return 1; }
  static Carry<R> step(Carry<R> c, V3<R>, const R* p) { return primitive_step(c, p[0]); }
  static R finalize(Carry<R> c) {
    const V3<R> q = vabs(c.z) - V3<R>(R(1));
    const R outside = len(vmax(q, R(0)));
    const R inside = std::fmin(std::fmax(q.x, std::fmax(q.y, q.z)), R(0));
    return (outside + inside) / std::fmax(std::fabs(c.dr), R(1e-6));
  }
};

// The formula image of an `// @image` formula (the image sampler, tpl:1111-1191):
// host texels of 4 words each (u16 R, G | u16 B, A | u8 near-slope codes | u8
// far-slope codes), set by oracle_set_image; empty: no image (size 0).
struct OracleImage {
  std::vector<uint32_t> texels;
  uint32_t w = 0, h = 0;
  float slope[4] = {0, 0, 0, 0};
};
inline OracleImage& oracle_image() {
  static OracleImage img;
  return img;
}

template <class R> struct ImageSampleR {
  R value[4], near[4], far[4];
};
// image_slope_decode (tpl:1164-1168)
template <class R> void slope_decode(uint32_t packed, R out[4]) {
  for (int k = 0; k < 4; ++k) {
    const R c = R((packed >> (8 * k)) & 0xffu);
    out[k] = c == R(0) ? R(0) : R(std::exp2((c - R(255)) / R(16) + R(1)));
  }
}
// image_texel (tpl:1170-1176)
template <class R> ImageSampleR<R> image_texel_r(const OracleImage& im, uint32_t x, uint32_t y) {
  const uint32_t* t = &im.texels[size_t(y * im.w + x) * 4];
  ImageSampleR<R> s;
  const R scale = R(1.0f / 65535.0f);
  const uint32_t ch[4] = {t[0] & 0xffffu, t[0] >> 16, t[1] & 0xffffu, t[1] >> 16};
  for (int k = 0; k < 4; ++k) s.value[k] = R(ch[k]) * scale;
  slope_decode<R>(t[2], s.near);
  slope_decode<R>(t[3], s.far);
  return s;
}
template <class R> ImageSampleR<R> image_mix_r(const ImageSampleR<R>& a, const ImageSampleR<R>& b, R t) {
  ImageSampleR<R> o;
  for (int k = 0; k < 4; ++k) {
    o.value[k] = a.value[k] * (R(1) - t) + b.value[k] * t;
    o.near[k] = a.near[k] * (R(1) - t) + b.near[k] * t;
    o.far[k] = a.far[k] * (R(1) - t) + b.far[k] * t;
  }
  return o;
}
// image_sample (tpl:1182-1191): bilinear, clamped at the edges
template <class R> ImageSampleR<R> image_sample_r(const OracleImage& im, R u, R v) {
  const uint32_t lx = im.w - 1, ly = im.h - 1;
  const R tx = std::fmin(std::fmax(u * R(im.w) - R(0.5), R(0)), R(lx));
  const R ty = std::fmin(std::fmax(v * R(im.h) - R(0.5), R(0)), R(ly));
  const uint32_t x0 = std::min(uint32_t(tx), lx), y0 = std::min(uint32_t(ty), ly);
  const uint32_t x1 = std::min(x0 + 1, lx), y1 = std::min(y0 + 1, ly);
  const R fx = tx - R(x0), fy = ty - R(y0);
  const ImageSampleR<R> top = image_mix_r(image_texel_r<R>(im, x0, y0), image_texel_r<R>(im, x1, y0), fx);
  const ImageSampleR<R> bottom = image_mix_r(image_texel_r<R>(im, x0, y1), image_texel_r<R>(im, x1, y1), fx);
  return image_mix_r(top, bottom, fy);
}

// Height map: formulas/heightmap_primitive.wgsl:14-62 with the image sampler above.
template <class R> struct HeightMap {
  static int iterations(const R*) { return 1; }  // primitive_de_iterations (tpl:1096)
  static R dot4(const R a[4], const R b[4]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3]; }
  static Carry<R> step(Carry<R> c, V3<R>, const R* p) {
    const R size = std::fmax(p[0], R(1e-4));
    const V3<R> q = c.z / (size * std::fmax(std::fabs(c.dr), R(1e-6)));
    const R lift = p[1];
    const R base = std::fmax(p[2], R(0));
    const bool up = lift >= R(0);
    const R w[4] = {p[3], p[4], p[5], p[6]};
    R k[4];
    if (p[7] > R(0.5)) {
      k[0] = -w[0]; k[1] = -w[1]; k[2] = -w[2];
      const R one[4] = {1, 1, 1, 1};
      k[3] = dot4(w, one);
    } else {
      for (int i = 0; i < 4; ++i) k[i] = w[i];
    }
    const OracleImage& im = oracle_image();
    R halfx = 1, halfy = 1, texel = 0, h_lo = 0, h_hi = 0;
    ImageSampleR<R> s;
    for (int i = 0; i < 4; ++i) s.value[i] = s.near[i] = s.far[i] = R(0);
    R slope[4] = {0, 0, 0, 0};
    if (im.w > 0 && im.h > 0 && !im.texels.empty()) {
      for (int i = 0; i < 4; ++i) slope[i] = R(im.slope[i]);
      const R dx = R(im.w), dy = R(im.h), m = std::fmax(dx, dy);
      halfx = dx / m;
      halfy = dy / m;
      texel = R(2) / m;
      s = image_sample_r<R>(im, q.x / halfx * R(0.5) + R(0.5), q.z / halfy * R(0.5) + R(0.5));
      h_lo = std::fmin(R(0), k[3] + (std::fmin(k[0], R(0)) + std::fmin(k[1], R(0)) + std::fmin(k[2], R(0))));
      h_hi = std::fmax(R(0), k[3] + (std::fmax(k[0], R(0)) + std::fmax(k[1], R(0)) + std::fmax(k[2], R(0))));
    }
    const R top = lift * dot4(k, s.value);
    const R dyv = up ? q.y - top : top - q.y;
    const R flat_side = up ? -base - q.y : q.y - base;
    const R ak[4] = {std::fabs(k[0]), std::fabs(k[1]), std::fabs(k[2]), std::fabs(k[3])};
    const R per_texel = std::fabs(lift) / std::fmax(texel, R(1e-6));
    const R g[3] = {per_texel * dot4(ak, slope), per_texel * dot4(ak, s.near), per_texel * dot4(ak, s.far)};
    R cc[3];
    for (int i = 0; i < 3; ++i) cc[i] = dyv / std::sqrt(R(1) + g[i] * g[i]);
    const R nearw = R(8) * texel, farw = R(64) * texel;  // IMAGE_SLOPE_RADIUS_NEAR / _FAR
    const R c_near = std::fmin(std::fmax(cc[1], -nearw), nearw);
    const R c_far = std::fmin(std::fmax(cc[2], -farw), farw);
    const R curved = dyv >= R(0) ? std::fmax(cc[0], std::fmax(c_near, c_far)) : std::fmin(cc[0], std::fmin(c_near, c_far));
    const R t_min = std::fmin(lift * h_lo, lift * h_hi), t_max = std::fmax(lift * h_lo, lift * h_hi);
    const R lo = up ? -base : std::fmin(t_min, base);
    const R hi = up ? std::fmax(t_max, -base) : base;
    const V3<R> e(std::fabs(q.x) - halfx, std::fmax(lo - q.y, q.y - hi), std::fabs(q.z) - halfy);
    const R bounds = len(vmax(e, R(0))) + std::fmin(std::fmax(e.x, std::fmax(e.y, e.z)), R(0));
    const R d = std::fmax(std::fmax(curved, flat_side), bounds);
    const R elevation = std::fmin(std::fmax((q.y - lo) / std::fmax(hi - lo, R(1e-4)), R(0)), R(1));
    return Carry<R>{V3<R>(R(0), elevation, R(0)), d * size};
  }
  static R finalize(Carry<R> c) { return c.dr; }
};

enum FormulaKind { F_MANDELBULB = 0, F_MANDELBOX, F_MENGER3, F_PSEUDOKLEINIAN, F_SPHERE, F_CUBE, F_HEIGHTMAP, F_COUNT };

inline int formula_index(const char* name) {
  const std::string n(name ? name : "");
  if (n == "mandelbrot") return F_MANDELBULB;
  if (n == "amazingbox_box") return F_MANDELBOX;
  if (n == "menger3_ifs") return F_MENGER3;
  if (n == "pseudokleinian_kleinian") return F_PSEUDOKLEINIAN;
  if (n == "sphere_primitive") return F_SPHERE;
  if (n == "cube_primitive") return F_CUBE;
  if (n == "heightmap_primitive") return F_HEIGHTMAP;
  return -1;
}

// ------------------------------------------------------------------ orbit trap
// OrbitTrap and its accumulator: tpl:1193-1289.
template <class R> R trap_distance(const nd_trap_desc& t, V3<R> z) {
  const V3<R> q = z - V3<R>(R(t.center[0]), R(t.center[1]), R(t.center[2]));
  switch (t.shape) {
    case ND_TRAP_SPHERE: return std::fabs(len(q) - R(t.radius));
    case ND_TRAP_BOX: {
      const V3<R> e = vabs(q) - V3<R>(R(t.box[0]), R(t.box[1]), R(t.box[2]));
      return std::fabs(len(vmax(e, R(0))) + std::fmin(std::fmax(e.x, std::fmax(e.y, e.z)), R(0)));
    }
    case ND_TRAP_CROSS: return std::fmin(std::fabs(q.x), std::fmin(std::fabs(q.y), std::fabs(q.z)));
    case ND_TRAP_TORUS: {
      const R a = std::sqrt(q.x * q.x + q.z * q.z) - R(t.radius);
      return std::fabs(std::sqrt(a * a + q.y * q.y) - R(t.tube));
    }
    default: return len(q);
  }
}

template <class R> struct TrapAcc {
  R x, y, z, w;
};

template <class R> TrapAcc<R> trap_begin(const nd_trap_desc& t) {
  const bool high = t.mode != ND_TRAP_MAX && t.mode != ND_TRAP_AVERAGE;
  return TrapAcc<R>{high ? R(1e6) : R(0), R(0), R(0), R(1e6)};
}

template <class R> void trap_update(TrapAcc<R>& a, const nd_trap_desc& t, V3<R> z, V3<R> zp, int it) {
  const R d = trap_distance(t, z);
  a.w = d;
  if (t.mode == ND_TRAP_MAX) {
    a.x = std::fmax(a.x, d);
  } else if (t.mode == ND_TRAP_AVERAGE) {
    if (z.x != zp.x || z.y != zp.y || z.z != zp.z) {
      a.x += d;
      a.y += R(1);
    }
  } else if (t.mode == ND_TRAP_ITERATION) {
    if (d < a.x) {
      a.x = d;
      a.z = R(it);
    }
  } else {
    a.x = std::fmin(a.x, d);
  }
}

template <class R> R trap_finish(const TrapAcc<R>& a, const nd_trap_desc& t, int iters) {
  if (t.mode == ND_TRAP_AVERAGE) return a.y > R(0.5) ? a.x / std::fmax(a.y, R(1)) : a.w;
  if (t.mode == ND_TRAP_LAST) return a.w;
  if (t.mode == ND_TRAP_ITERATION) return (a.z + R(1)) / R(std::max(iters, 1));
  return a.x;
}

// ------------------------------------------------------------------ one DE evaluation
template <class R> struct DE {
  R d;
  R trap;
  int iters;  // iterations in which the carry changed
};

// The generated per-formula wrapper formula_N (fractal_renderer.zig:490-512) with
// the single-instance scene_de (tpl:1756-1779): instance_local is the identity and
// instance_de_factor = min(scale) * clamp(step_safety, 0.001, 1) (tpl:1611-1620).
// Iteration counts are capped at 4096 (a build-wide watchdog cap).
template <class R, class F> DE<R> formula_de(V3<R> pos, const R* p, const nd_trap_desc& trap, R factor) {
  Carry<R> c{pos, R(1)};
  TrapAcc<R> acc = trap_begin<R>(trap);
  int n = F::iterations(p);
  if (n > 4096) n = 4096;
  int changed = 0;
  for (int it = 0; it < n; ++it) {
    const V3<R> zp = c.z;
    c = F::step(c, pos, p);
    if (c.z.x != zp.x || c.z.y != zp.y || c.z.z != zp.z) ++changed;
    trap_update(acc, trap, c.z, zp, it);
  }
  DE<R> out;
  out.d = F::finalize(c) * factor;
  out.trap = trap_finish(acc, trap, n);
  out.iters = changed;
  return out;
}

template <class R> DE<R> eval_de(int kind, V3<R> pos, const R* p, const nd_trap_desc& trap, R factor) {
  switch (kind) {
    case F_MANDELBULB: return formula_de<R, Mandelbulb<R>>(pos, p, trap, factor);
    case F_MANDELBOX: return formula_de<R, Mandelbox<R>>(pos, p, trap, factor);
    case F_MENGER3: return formula_de<R, Menger3<R>>(pos, p, trap, factor);
    case F_PSEUDOKLEINIAN: return formula_de<R, PseudoKleinian<R>>(pos, p, trap, factor);
    case F_SPHERE: return formula_de<R, SpherePrim<R>>(pos, p, trap, factor);
    case F_HEIGHTMAP: return formula_de<R, HeightMap<R>>(pos, p, trap, factor);
    default: return formula_de<R, CubePrim<R>>(pos, p, trap, factor);
  }
}

// eval_step / eval_finalize dispatch (fractal_renderer.zig:529-534).
template <class R> Carry<R> step_kind(int kind, Carry<R> c, V3<R> pos, const R* p) {
  switch (kind) {
    case F_MANDELBULB: return Mandelbulb<R>::step(c, pos, p);
    case F_MANDELBOX: return Mandelbox<R>::step(c, pos, p);
    case F_MENGER3: return Menger3<R>::step(c, pos, p);
    case F_PSEUDOKLEINIAN: return PseudoKleinian<R>::step(c, pos, p);
    case F_SPHERE: return SpherePrim<R>::step(c, pos, p);
    case F_HEIGHTMAP: return HeightMap<R>::step(c, pos, p);
    default: return CubePrim<R>::step(c, pos, p);
  }
}
template <class R> R finalize_kind(int kind, Carry<R> c) {
  switch (kind) {
    case F_MANDELBULB: return Mandelbulb<R>::finalize(c);
    case F_MANDELBOX: return Mandelbox<R>::finalize(c);
    case F_MENGER3: return Menger3<R>::finalize(c);
    case F_PSEUDOKLEINIAN: return PseudoKleinian<R>::finalize(c);
    case F_SPHERE: return SpherePrim<R>::finalize(c);
    case F_HEIGHTMAP: return HeightMap<R>::finalize(c);
    default: return CubePrim<R>::finalize(c);
  }
}

// ------------------------------------------------------------------ scenes
// Smooth combine family (tpl:1648-1706): k <= 1e-4 is the hard operation.
template <class R> R mixr(R a, R b, R h) { return a * (R(1) - h) + b * h; }
template <class R> R s_min(R a, R b, R k) {
  if (k <= R(0.0001)) return std::fmin(a, b);
  const R h = clampv(R(0.5) + R(0.5) * (b - a) / k, R(0), R(1));
  return mixr(b, a, h) - k * h * (R(1) - h);
}
template <class R> R s_max(R a, R b, R k) {
  if (k <= R(0.0001)) return std::fmax(a, b);
  const R h = clampv(R(0.5) - R(0.5) * (b - a) / k, R(0), R(1));
  return mixr(b, a, h) + k * h * (R(1) - h);
}
template <class R> R s_sub(R cut, R base, R k) {
  if (k <= R(0.0001)) return std::fmax(-cut, base);
  const R h = clampv(R(0.5) - R(0.5) * (base + cut) / k, R(0), R(1));
  return mixr(base, -cut, h) + k * h * (R(1) - h);
}
template <class R> R s_min_lin(R a, R b, R k) {
  if (k <= R(0.0001)) return std::fmin(a, b);
  return std::fmin(b - std::fmax(k - a, R(0)), a - std::fmax(k - b, R(0)));
}
template <class R> R s_min_nlin(R a, R b, R k) {
  if (k <= R(0.0001)) return std::fmin(a, b);
  const R ra = std::fmax(k - a, R(0)), rb = std::fmax(k - b, R(0));
  return std::fmin(b - ra * (k - rb) / k, a - rb * (k - ra) / k);
}
template <class R> R s_mix(R a, R b, R k) {
  if (k <= R(0.0001)) return std::fmin(a, b);
  const R h = clampv(R(0.5) + R(0.5) * (b - a) / k, R(0), R(1));
  return mixr(b, a, h);
}
// combine_de (tpl:1708-1730): d is the scene so far, di the next instance.
template <class R> R combine(int mode, R d, R di, R k) {
  switch (mode) {
    case ND_COMBINE_UNION: return std::fmin(d, di);
    case ND_COMBINE_SMOOTH_MIN: return s_min(d, di, k);
    case ND_COMBINE_SMOOTH_MAX: return s_max(d, di, k);
    case ND_COMBINE_SMOOTH_INV_MAX: return s_sub(di, d, k);
    case ND_COMBINE_SMOOTH_MIN_LIN: return s_min_lin(d, di, k);
    case ND_COMBINE_SMOOTH_MIN_NLIN: return s_min_nlin(d, di, k);
    default: return s_mix(d, di, k);
  }
}

// combine_de's material weight (tpl:1708-1730): the share of the scene so far.
template <class R> R combine_weight(int mode, R d, R di, R k) {
  const bool hard = k <= R(0.0001);
  const R closer = di < d ? R(0) : R(1);
  switch (mode) {
    case ND_COMBINE_SMOOTH_MIN:
    case ND_COMBINE_SMOOTH_MIX: return hard ? closer : clampv(R(0.5) + R(0.5) * (di - d) / k, R(0), R(1));
    case ND_COMBINE_SMOOTH_MAX: return hard ? (di > d ? R(0) : R(1)) : clampv(R(0.5) - R(0.5) * (di - d) / k, R(0), R(1));
    case ND_COMBINE_SMOOTH_INV_MAX:
      return hard ? (-di > d ? R(0) : R(1)) : R(1) - clampv(R(0.5) - R(0.5) * (d + di) / k, R(0), R(1));
    default: return closer;
  }
}

// orbit_trap_to_strip (tpl:2025-2035): TRAP_MIN_SPAN 1e-4; repeat 1 fract, 2 mirror.
template <class R> R trap_strip(R span, R offset, int repeat, R v) {
  const R x = v / std::fmax(span, R(1e-4)) + offset;
  if (repeat == 1) return x - std::floor(x);
  if (repeat == 2) return R(1) - std::fabs((x * R(0.5) - std::floor(x * R(0.5))) * R(2) - R(1));
  return clampv(x, R(0), R(1));
}

// The lite material at a strip position: sample_gradient (tpl:2003-2023) with
// mix_material's blend (tpl:1980-2001) of colour, glossiness and ior; no stops:
// default_material (tpl:1965-1977).  out: r, g, b, glossiness, ior.
inline void lite_stop_material(const nd_lite_desc& L, double strip, double out[5]) {
  auto take = [&](const nd_color_stop& c) {
    for (int k = 0; k < 3; ++k) out[k] = c.color[k];
    out[3] = c.glossiness;
    out[4] = c.ior;
  };
  out[0] = 0.8; out[1] = 0.8; out[2] = 0.85; out[3] = 0.3; out[4] = 1.5;
  const int count = std::min(L.color_count, ND_MAX_COLOR_STOPS);
  if (count <= 0) return;
  if (count == 1 || strip <= L.colors[0].position) return take(L.colors[0]);
  if (strip >= L.colors[count - 1].position) return take(L.colors[count - 1]);
  take(L.colors[count - 1]);
  for (int i = 0; i < count - 1; ++i) {
    const nd_color_stop& a = L.colors[i];
    const nd_color_stop& b = L.colors[i + 1];
    if (strip >= a.position && strip <= b.position) {
      const double f = (strip - a.position) / std::max(double(b.position) - a.position, 1e-4);
      for (int k = 0; k < 3; ++k) out[k] = b.color[k] + (a.color[k] - b.color[k]) * (1.0 - f);
      out[3] = b.glossiness + (a.glossiness - b.glossiness) * (1.0 - f);
      out[4] = b.ior + (a.ior - b.ior) * (1.0 - f);
      return;
    }
  }
}

// scene_de (tpl:1756-1779) over an nd_scene_desc: per instance the inverse placement
// (instance_local tpl:1597-1609: rotation frame, then per-axis signed scale with
// |s| >= 0.001), the DE factor min|s| * clamp(step_safety, 0.001, 1)
// (tpl:1611-1620), hybrid mixins (eval_mixed tpl:1335-1392), then the carves
// (apply_carves tpl:1741-1753, blend 0.2 r).  The trap and iteration count are those
// of the visible instance with the smallest DE.  kind / mkind hold oracle formula
// kinds for the instances' and mixins' formula ids.
template <class R> struct SceneEval {
  const nd_scene_desc* scene = nullptr;
  int kind[ND_MAX_INSTANCES] = {0, 0, 0, 0};
  int mkind[ND_MAX_INSTANCES][ND_MAX_MIXINS] = {};
  double max_dist = 0;

  DE<R> mixed(const nd_instance_desc& in, int slot, V3<R> pos) const {
    R p[ND_MAX_PARAMS], mp[ND_MAX_MIXINS][ND_MAX_PARAMS];
    for (int k = 0; k < ND_MAX_PARAMS; ++k) p[k] = R(in.params[k]);
    for (int j = 0; j < ND_MAX_MIXINS; ++j)
      for (int k = 0; k < ND_MAX_PARAMS; ++k) mp[j][k] = R(in.mixins[j].params[k]);
    const int base_n = std::max(in.hybrid_base_iters, 0);
    const int mixins = std::min(std::max(in.mixin_count, 0), ND_MAX_MIXINS);
    int cycle = base_n;
    for (int j = 0; j < mixins; ++j) cycle += std::max(in.mixins[j].iterations, 0);
    cycle = std::max(cycle, 1);
    const int total = std::min(std::max(in.hybrid_total_iters, 0), 4096);
    Carry<R> c{pos, R(1)};
    TrapAcc<R> acc = trap_begin<R>(in.trap);
    int changed = 0;
    for (int it = 0; it < total; ++it) {
      int at = it % cycle;
      int k = kind[slot];
      const R* pp = p;
      bool have = true;
      if (at >= base_n) {  // hybrid_step: which mixin owns this iteration
        at -= base_n;
        have = false;
        for (int j = 0; j < mixins; ++j) {
          const int nj = std::max(in.mixins[j].iterations, 0);
          if (at < nj) {
            k = mkind[slot][j];
            pp = mp[j];
            have = true;
            break;
          }
          at -= nj;
        }
      }
      const V3<R> zp = c.z;
      if (have) c = step_kind(k, c, pos, pp);
      if (c.z.x != zp.x || c.z.y != zp.y || c.z.z != zp.z) ++changed;
      trap_update(acc, in.trap, c.z, zp, it);
    }
    DE<R> o;
    o.d = finalize_kind(kind[slot], c);
    o.trap = trap_finish(acc, in.trap, total);
    o.iters = changed;
    return o;
  }

  DE<R> instance(int slot, V3<R> pos) const {
    const nd_instance_desc& in = scene->instances[slot];
    R s[3], mag_min = R(1e30);
    for (int i = 0; i < 3; ++i) {
      const R mag = std::fmax(std::fabs(R(in.scale[i])), R(0.001));
      s[i] = in.scale[i] < 0.0f ? -mag : mag;
      mag_min = std::fmin(mag_min, mag);
    }
    const R factor = mag_min * clampv(R(in.step_safety), R(0.001), R(1));
    const V3<R> d = pos - V3<R>(R(in.offset[0]), R(in.offset[1]), R(in.offset[2]));
    R f[9];  // frame columns: local_i = (column_i . d) / s_i
    for (int i = 0; i < 9; ++i) f[i] = R(in.frame[i]);
    const V3<R> local((f[0] * d.x + f[1] * d.y + f[2] * d.z) / s[0], (f[3] * d.x + f[4] * d.y + f[5] * d.z) / s[1],
                      (f[6] * d.x + f[7] * d.y + f[8] * d.z) / s[2]);
    DE<R> o;
    if (in.mixin_count > 0) {
      o = mixed(in, slot, local);
    } else {
      R p[ND_MAX_PARAMS];
      for (int k = 0; k < ND_MAX_PARAMS; ++k) p[k] = R(in.params[k]);
      o = eval_de<R>(kind[slot], local, p, in.trap, R(1));
    }
    o.d = o.d * factor;
    return o;
  }

  // hit_material (tpl:2128-2155) for the lite pass: each visible instance's
  // material at its own trap strip, blended with combine_de's weight; colors: the
  // scene's ND_MAX_INSTANCES descriptors.  out: r, g, b, glossiness, ior.
  void material(V3<R> pos, const nd_lite_desc* colors, double out[5]) const {
    lite_stop_material(nd_lite_desc(), 0.0, out);
    R d = R(0);
    bool first = true;
    const int count = std::min(std::max(scene->instance_count, 1), ND_MAX_INSTANCES);
    for (int i = 0; i < count; ++i) {
      const nd_instance_desc& in = scene->instances[i];
      if (in.hidden) continue;
      const DE<R> di = instance(i, pos);
      double mi[5];
      lite_stop_material(colors[i], trap_strip<double>(in.trap.span, in.trap.offset, in.trap.repeat, double(di.trap)),
                         mi);
      if (first) {
        d = di.d;
        for (int k = 0; k < 5; ++k) out[k] = mi[k];
        first = false;
        continue;
      }
      const double h = double(combine_weight<R>(in.combine_mode, d, di.d, R(in.blend_k)));
      for (int k = 0; k < 5; ++k) out[k] = mi[k] * (1.0 - h) + out[k] * h;
      d = combine<R>(in.combine_mode, d, di.d, R(in.blend_k));
    }
  }

  DE<R> de(V3<R> pos) const {
    const R empty = R(float(max_dist) * 2.0f + 1.0f);  // empty_scene_de
    DE<R> o{empty, R(0), 0};
    R d = empty, best = R(0);
    bool first = true;
    const int count = std::min(std::max(scene->instance_count, 1), ND_MAX_INSTANCES);
    for (int i = 0; i < count; ++i) {
      const nd_instance_desc& in = scene->instances[i];
      if (in.hidden) continue;
      const DE<R> di = instance(i, pos);
      if (first || di.d < best) {
        best = di.d;
        o.trap = di.trap;
        o.iters = di.iters;
      }
      d = first ? di.d : combine<R>(in.combine_mode, d, di.d, R(in.blend_k));
      first = false;
    }
    if (first) return DE<R>{empty, R(0), 0};
    const int carves = std::min(std::max(scene->carve_count, 0), ND_MAX_CARVES);
    for (int i = 0; i < carves; ++i) {
      const float* c = scene->carves[i];
      const R r = R(c[3]);
      const R l = len(pos - V3<R>(R(c[0]), R(c[1]), R(c[2])));
      d = s_sub(l - r, d, R(0.2) * r);
    }
    o.d = d;
    return o;
  }
};

// ------------------------------------------------------------------ empty-space accelerator
// Cascade placement (placeCascades, src/gpu/accel.zig:32-56, clampResolution :28-31),
// the grid build (cs_build_accel tpl:5412-5431) and the lookup (accel_skip
// tpl:428-447), in f32 like the reference; grid layout [level][z][y][x].
constexpr int kAccelMaxCascades = 8;  // MAX_CASCADES tpl:31
inline int accel_clamp_res(int res) { return std::min(std::max(res, 16), 160) / 4 * 4; }
inline int accel_clamp_levels(int levels) { return std::min(std::max(levels, 1), kAccelMaxCascades); }

struct AccelGrid {
  int res = 0, levels = 0;
  float prm[kAccelMaxCascades][4] = {};  // corner xyz, cell size
  std::vector<float> v;

  void place(const double cam[3], float max_dist, int nlevels, int nres) {
    res = nres;
    levels = nlevels;
    const float res_f = float(std::max(res, 1));
    const float coarsest = std::fmax(2.0f * max_dist / res_f, 1e-6f);
    for (int l = 0; l < levels; ++l) {
      const float cell = coarsest / float(1u << (levels - 1 - l));
      const float half = 0.5f * res_f * cell;
      for (int a = 0; a < 3; ++a) prm[l][a] = std::floor((float(cam[a]) - half) / cell) * cell;
      prm[l][3] = cell;
    }
  }

  // de(V3<float> centre) -> distance (any float type); safe skip per voxel centre
  template <class F> void build(float safety, int nthreads, F&& de) {
    const int64_t r = res, total = int64_t(levels) * r * r * r;
    v.assign(size_t(total), 0.0f);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 256)
    for (int64_t idx = 0; idx < total; ++idx) {
      const int64_t x = idx % r, y = (idx / r) % r, gz = idx / (r * r);
      const int l = int(gz / r);
      const int64_t z = gz % r;
      const float cell = prm[l][3];
      const V3<float> c(prm[l][0] + (float(x) + 0.5f) * cell, prm[l][1] + (float(y) + 0.5f) * cell,
                        prm[l][2] + (float(z) + 0.5f) * cell);
      const float d = float(de(c));
      v[size_t(idx)] = std::fmax(d - 0.8660254f * cell, 0.0f) * safety;  // HALF_SQRT3 tpl:62
    }
  }

  float skip(float px, float py, float pz) const {
    for (int l = 0; l < levels; ++l) {
      const float cell = prm[l][3];
      if (!(cell > 0.0f)) continue;
      const float fx = std::floor((px - prm[l][0]) / cell);
      const float fy = std::floor((py - prm[l][1]) / cell);
      const float fz = std::floor((pz - prm[l][2]) / cell);
      const float rf = float(res);
      if (!(fx >= 0.0f && fy >= 0.0f && fz >= 0.0f && fx < rf && fy < rf && fz < rf)) continue;
      return v[((size_t(l) * res + size_t(fz)) * res + size_t(fy)) * res + size_t(fx)];
    }
    return 0.0f;
  }
};

// fresnel_schlick (tpl:3424-3430)
template <class R> R fresnel_schlick(R cos_theta, R ior) {
  const R r0root = (R(1) - ior) / (R(1) + ior);
  const R r0 = r0root * r0root;
  const R c = clampv(R(1) - std::fabs(cos_theta), R(0), R(1));
  const R c2 = c * c;
  return r0 + (R(1) - r0) * c2 * c2 * c;
}

// ------------------------------------------------------------------ per-ray result
struct RayOut {
  double depth;       // t at the hit, 0 on a miss
  double normal[3];
  int hit;
  double trap;
  uint32_t steps;
  uint32_t iters;
  double shade;
  double shadow;
  uint32_t evals;
  double margin;      // smallest |d - eps| / eps over all hit decisions of the primary march
};

// Philox-free counter hash for jitter: SplitMix64 of (seed, key) -> two floats in
// [0, 1) with 24-bit resolution, key = (sample * height + row) * width + column of
// the ray in the whole frame.  The CUDA library uses the same function.
inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
inline void jitter2(uint64_t seed, uint64_t ray, double* jx, double* jy) {
  const uint64_t h = splitmix64(seed ^ splitmix64(ray));
  *jx = double(uint32_t(h) >> 8) * (1.0 / 16777216.0);
  *jy = double(uint32_t(h >> 32) >> 8) * (1.0 / 16777216.0);
}

template <class R> struct Tracer {
  const nd_view_desc& v;
  int kind;
  R p[ND_MAX_PARAMS];
  R factor;
  V3<double> org;
  uint32_t evals = 0;
  double de_scale = 1.0;  // every DE value is multiplied by this (stability probes)
  const SceneEval<R>* scene = nullptr;  // a multi-instance scene instead of the view's formula
  const AccelGrid* accel = nullptr;     // the view's empty-space accelerator, when it has one
  const nd_lite_desc* scene_colors = nullptr;  // lite pass: the scene instances' colour stops

  Tracer(const nd_view_desc& view, int k) : v(view), kind(k) {
    for (int i = 0; i < ND_MAX_PARAMS; ++i) p[i] = R(view.params[i]);
    factor = R(std::min(std::max(double(view.step_safety), 0.001), 1.0));
    org = V3<double>(view.cam_pos[0], view.cam_pos[1], view.cam_pos[2]);
  }

  DE<R> de_at(V3<double> pos) {
    ++evals;
    const V3<R> q(R(pos.x), R(pos.y), R(pos.z));
    DE<R> o = scene ? scene->de(q) : eval_de<R>(kind, q, p, v.trap, factor);
    if (de_scale != 1.0) o.d = R(double(o.d) * de_scale);
    return o;
  }

  // march_epsilon: tpl:1813-1815
  double eps(double t) const { return double(R(v.eps_coef) * R(t) + R(v.eps_floor)); }

  // march_to: tpl:1859-1963, without the accelerator, warps, coarse mode and the
  // overstep diagnostic (all off on this path).  t, lo, hi are kept in double.
  void march(V3<double> dir, RayOut& o, DE<R>& hit_de) {
    const int max_steps = v.max_steps;
    const bool hq = v.high_quality != 0;
    const int budget = std::max(v.refine_budget, 0);
    const bool on_hit = v.march_verify == 0;
    const int refine_budget = on_hit ? 0 : budget;
    const int bisect_budget = on_hit ? budget : 0;
    const double footprint = double(v.hq_footprint_px) * 2.0 / std::max(double(v.height), 1.0);
    const double max_t = v.max_dist;
    double t = 0, lo = 0, hi = 0;
    int i = 0, refines = 0;
    bool probing = true, bisecting = false, resolved = false;
    o.margin = 1e30;
    const long max_samples = long(max_steps) * (1 + refine_budget) + bisect_budget;
    for (long n = 0; n < max_samples; ++n) {
      const double st = probing ? t : 0.5 * (lo + hi);
      const double e = eps(st);
      const V3<double> pos = org + dir * st;
      if (probing && accel) {
        // accel_skip before the DE (march_to tpl:1890-1900): a safe jump costs no evaluation
        const double skip = double(accel->skip(float(pos.x), float(pos.y), float(pos.z)));
        if (skip > e) {
          lo = st;
          t = st + skip;
          ++i;
          o.margin = std::min(o.margin, std::fabs(t - max_t) / max_t);
          if (t > max_t || i >= max_steps) break;
          continue;
        }
      }
      const DE<R> de = de_at(pos);
      const double d = double(de.d);
      o.margin = std::min(o.margin, std::fabs(d - e) / std::max(e, 1e-30));
      if (bisecting) {
        if (d < e) {
          hi = st;
          hit_de = de;
        } else {
          lo = st;
        }
        ++refines;
        if (hi - lo <= e || refines >= bisect_budget) {
          o.hit = 1; o.depth = hi; o.steps = uint32_t(i);
          return;
        }
        continue;
      }
      if (d < e) {
        if (on_hit && bisect_budget > 0 && st - lo > e) {
          bisecting = true;
          probing = false;
          hi = st;
          refines = 0;
          hit_de = de;
          continue;
        }
        o.hit = 1; o.depth = st; o.steps = uint32_t(i);
        hit_de = de;
        return;
      }
      if (probing) {
        lo = t;
        hi = t + d;
        refines = 0;
        resolved = false;
        probing = false;
      } else {
        if (d >= hi - st) resolved = true;
        else hi = st;
        ++refines;
      }
      if (resolved || refines >= refine_budget) {
        if (hq && !resolved && refine_budget > 0) hi = std::min(hi, lo + std::max(t, 1.0) * footprint);
        t = hi;
        ++i;
        o.margin = std::min(o.margin, std::fabs(t - max_t) / max_t);
        if (t > max_t || i >= max_steps) break;
        probing = true;
      }
    }
    o.hit = 0; o.depth = t; o.steps = uint32_t(max_steps);
  }

  // Normals: tetrahedral gradient with e = eps(t) (estimate_normal / tetra_gradient
  // tpl:1783-1804), or 6-tap central differences with h = coef * t.
  V3<double> normal(V3<double> pos, double t) {
    V3<double> g(0.0);
    if (v.normal_mode == ND_NORMAL_CENTRAL) {
      const double h = v.normal_h_coef > 0 ? double(v.normal_h_coef) * t : eps(t);
      for (int a = 0; a < 3; ++a) {
        V3<double> k(0.0);
        (a == 0 ? k.x : a == 1 ? k.y : k.z) = h;
        const double dp = double(de_at(pos + k).d);
        const double dm = double(de_at(pos - k).d);
        (a == 0 ? g.x : a == 1 ? g.y : g.z) = dp - dm;
      }
    } else {
      const double e = eps(t);
      const V3<double> ks[4] = {V3<double>(1, -1, -1), V3<double>(-1, -1, 1), V3<double>(-1, 1, -1), V3<double>(1, 1, 1)};
      for (int i = 0; i < 4; ++i) g = g + ks[i] * double(de_at(pos + ks[i] * e).d);
    }
    const double l = len(g);
    return l > 0 ? g / l : g;
  }

  // Opaque soft shadow toward a LIGHT_GLOBAL light: shadow_factor tpl:2365-2375 and
  // visibility_march tpl:2282-2342 with constants tpl:2344-2353 (bias 0.004, hit
  // eps 5e-4, min step 1e-3, at most min(max_steps, 40) steps, light distance
  // 2 * max_dist as light_sample_ex gives for LIGHT_GLOBAL, tpl:2187-2190).
  double shadow(V3<double> pos, V3<double> n, V3<double> l) {
    const V3<double> o = pos + n * 0.004;
    const double light_dist = double(v.max_dist) * 2.0;
    const int steps = std::min(v.max_steps, 40);
    double t = 0.004, res = 1.0;
    for (int i = 0; i < steps; ++i) {
      if (t >= light_dist) break;
      const V3<double> p = o + l * t;
      if (accel) {  // visibility_march tpl:2297-2303
        const double skip = double(accel->skip(float(p.x), float(p.y), float(p.z)));
        if (skip > 0.001 && double(v.shadow_k) * skip >= res * t) {
          t += skip;
          continue;
        }
      }
      const double d = double(de_at(p).d);
      if (d < 0.0005) return 0.0;
      res = std::min(res, double(v.shadow_k) * d / t);
      t += std::max(d, 0.001);
    }
    return clampv(res, 0.0, 1.0);
  }

  // Primary ray direction of a work item (camera ray, see trace()).
  V3<double> ray_dir(int64_t ray) const {
    const int64_t npix = int64_t(v.tile_w) * v.tile_h;
    const int64_t s = ray / npix, pix = ray % npix;
    const int px = v.tile_x + int(pix % v.tile_w), py = v.tile_y + int(pix / v.tile_w);
    double jx = 0.5, jy = 0.5;
    // the jitter is keyed by the sample's place in the whole frame (sample, row,
    // column): a view cut into tiles draws the same rays as the view itself
    if (v.spp > 1) jitter2(v.seed, (uint64_t(s) * uint64_t(v.height) + uint64_t(py)) * uint64_t(v.width) + uint64_t(px),
                           &jx, &jy);
    const double ndc_x = 2.0 * (px + jx) / v.width - 1.0;
    const double ndc_y = 1.0 - 2.0 * (py + jy) / v.height;
    const double ux = ndc_x * double(v.width) / double(v.height), uy = -ndc_y;
    const V3<double> f(v.fwd[0], v.fwd[1], v.fwd[2]), r(v.right[0], v.right[1], v.right[2]),
        u(v.up[0], v.up[1], v.up[2]);
    return norm(f + r * ux + u * uy);
  }

  // Lite shading of a hit (shade_lite tpl:4424-4444): material from the colour strip
  // (orbit_trap_to_strip tpl:2025-2035, sample_gradient tpl:2003-2023 with
  // mix_material tpl:1980-2001, default_material tpl:1965-1977), ambient occlusion
  // (calc_ao tpl:1817-1840), point / global lights (light_sample_ex tpl:2178-2189),
  // Blinn-Phong with power mix(4, 128, glossiness) (tpl:3071-3072), times
  // 1 - fresnel_schlick (tpl:3424-3430).
  // calc_ao (tpl:1817-1840)
  double ao(V3<double> pos, V3<double> n, double t) {
    const double radius = clampv(t * 0.04, 0.003, 0.25);
    double occ = 0.0, w = 1.0;
    for (int i = 0; i < 5; ++i) {
      const double step = radius * (0.2 + 0.2 * i);
      const double d = double(de_at(pos + n * step).d);
      occ += std::max(step - d, 0.0) * w;
      w *= 0.6;
    }
    return clampv(1.0 - 2.0 * occ / radius, 0.0, 1.0);
  }

  void lite(const nd_lite_desc& L, int64_t ray, double t, V3<double> n, double trap, double* rgb) {
    const V3<double> dir = ray_dir(ray);
    const V3<double> pos = org + dir * t;
    double mat[5];
    if (scene && scene_colors) scene->material(V3<R>(R(pos.x), R(pos.y), R(pos.z)), scene_colors, mat);
    else lite_stop_material(L, trap_strip<double>(v.trap.span, v.trap.offset, v.trap.repeat, trap), mat);
    const double col[3] = {mat[0], mat[1], mat[2]}, gloss = mat[3], ior = mat[4];
    const double spec_power = 4.0 + (128.0 - 4.0) * clampv(gloss, 0.0, 1.0);
    const double fresnel = fresnel_schlick(dot(dir, n), std::max(ior, 1.0));
    const double occl = L.ambient_occlusion ? ao(pos, n, t) : 1.0;
    double diff[3] = {0.15 * occl, 0.15 * occl, 0.15 * occl}, spec[3] = {0, 0, 0};
    for (int i = 0; i < std::min(L.light_count, ND_MAX_LIGHTS); ++i) {
      const nd_light& l = L.lights[i];
      const V3<double> p(l.position_or_direction[0], l.position_or_direction[1], l.position_or_direction[2]);
      double lc[3] = {double(l.color[0]) * l.brightness, double(l.color[1]) * l.brightness,
                      double(l.color[2]) * l.brightness};
      V3<double> ld;
      if (l.type == ND_LIGHT_POINT) {
        const V3<double> tl = p - pos;
        const double dist = len(tl);
        ld = tl / std::max(dist, 1e-4);
        for (double& x2 : lc) x2 /= std::max(dist * dist, 0.01);
      } else {
        ld = norm(p);
      }
      const double ndotl = std::max(dot(n, ld), 0.0);
      if (ndotl <= 0.0) continue;
      for (int k = 0; k < 3; ++k) diff[k] += lc[k] * ndotl;
      if (L.specular) {
        const V3<double> h = norm(ld - dir);
        const double sp = std::pow(std::max(dot(n, h), 0.0), spec_power) * gloss;
        for (int k = 0; k < 3; ++k) spec[k] += lc[k] * sp;
      }
    }
    for (int k = 0; k < 3; ++k) rgb[k] = (1.0 - fresnel) * (col[k] * diff[k] + spec[k]);
  }

  RayOut trace(int64_t ray) {
    RayOut o;
    memset(&o, 0, sizeof(o));
    evals = 0;
    const int64_t npix = int64_t(v.tile_w) * v.tile_h;
    const int64_t s = ray / npix, pix = ray % npix;
    const int px = v.tile_x + int(pix % v.tile_w), py = v.tile_y + int(pix / v.tile_w);
    double jx = 0.5, jy = 0.5;
    if (v.spp > 1) jitter2(v.seed, (uint64_t(s) * uint64_t(v.height) + uint64_t(py)) * uint64_t(v.width) + uint64_t(px),
                           &jx, &jy);
    // camera ray: cs_wf_generate tpl:5120-5127 and fs_simple tpl:4523-4525; the tile
    // transform (fractal_renderer.zig:852-863) is folded into full-frame pixels.
    const double ndc_x = 2.0 * (px + jx) / v.width - 1.0;
    const double ndc_y = 1.0 - 2.0 * (py + jy) / v.height;
    const double aspect = double(v.width) / double(v.height);
    const double ux = ndc_x * aspect, uy = -ndc_y;
    const V3<double> f(v.fwd[0], v.fwd[1], v.fwd[2]), r(v.right[0], v.right[1], v.right[2]),
        u(v.up[0], v.up[1], v.up[2]);
    const V3<double> dir = norm(f + r * ux + u * uy);
    DE<R> hit_de{R(0), R(0), 0};
    march(dir, o, hit_de);
    o.shadow = 1.0;
    if (!o.hit) {
      o.depth = 0;
      o.evals = evals;
      return o;
    }
    o.trap = double(hit_de.trap);
    o.iters = uint32_t(hit_de.iters);
    const V3<double> pos = org + dir * o.depth;
    const V3<double> n = normal(pos, o.depth);
    o.normal[0] = n.x; o.normal[1] = n.y; o.normal[2] = n.z;
    // simple_geometry (tpl:4492-4507): key light normalize(-dir + 0.45 up - 0.35 right)
    // in camera space, or the view's directional light when one is given.
    V3<double> key;
    const V3<double> ld(v.light_dir[0], v.light_dir[1], v.light_dir[2]);
    if (v.shadow || dot(ld, ld) > 0) key = norm(ld);
    else key = norm(-dir + norm(u) * 0.45 - norm(r) * 0.35);
    if (v.shadow) o.shadow = shadow(pos, n, key);
    const double lam = std::max(dot(n, key), 0.0) * o.shadow;
    o.shade = 0.18 + (1.0 - 0.18) * lam;
    o.evals = evals;
    return o;
  }
};

}  // namespace oracle
