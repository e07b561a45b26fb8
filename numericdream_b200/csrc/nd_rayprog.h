// The ray program of the sphere-tracing pass, shared by the CUDA kernels
// (nd_kernels.cuh) and by the host op-counting build (nd_opcount.cpp).
//
// Work model.  A launch covers a list of views; every (view, sample, pixel) is one
// work item ("ray") with a global index; views are concatenated in call order and
// the G-buffer is indexed by that global index.
//
// Ray program.  The march of one ray is the reference's march_to
// (src/gpu/shaders/template.wgsl:1859-1963) followed by estimate_normal
// (tpl:1783-1804, or 6-tap central differences), the orbit trap of the DE
// evaluation at the hit (formula_N, src/gpu/fractal_renderer.zig:490-512) and an
// opaque soft shadow (visibility_march / shadow_factor, tpl:2282-2375).  In the
// persistent kernel the whole program is a state machine that spends exactly one DE
// evaluation per loop iteration, so all live lanes of a warp evaluate the DE
// together whatever phase (probe, bisection, normal tap, shadow step) each is in;
// lanes that finish are refilled with new rays once enough of them are idle.
//
// Precision: the DE runs in T (float by default); the ray origin, direction, t,
// the bisection interval and the normal/shadow sample positions are double.
#pragma once

#include <stdint.h>
#include <type_traits>

#include "nd_helpers.h"
#include "nd_dual.h"
#include "../../include/nd_march.h"
#if defined(__CUDACC__)
#include <cuda_fp16.h>
#endif

#if defined(__CUDACC__)
#define ND_DEV_INLINE __host__ __device__ __forceinline__
#else
#define ND_DEV_INLINE inline
#endif

namespace nd {

// Correctly rounded arithmetic that the compiler may not contract into FMAs.
#if defined(__CUDA_ARCH__)
ND_DEV_INLINE float rn_mul(float a, float b) { return __fmul_rn(a, b); }
ND_DEV_INLINE float rn_add(float a, float b) { return __fadd_rn(a, b); }
ND_DEV_INLINE double rn_mul(double a, double b) { return __dmul_rn(a, b); }
ND_DEV_INLINE double rn_add(double a, double b) { return __dadd_rn(a, b); }
ND_DEV_INLINE double fma_d(double a, double b, double c) { return __fma_rn(a, b, c); }
ND_DEV_INLINE float load_ro(const float* p) { return __ldg(p); }
ND_DEV_INLINE int32_t float_bits(float x) { return __float_as_int(x); }
ND_DEV_INLINE uint16_t half_bits(float x) { return __half_as_ushort(__float2half_rn(x)); }
#else
// host builds of this header are compiled with -ffp-contract=off
ND_DEV_INLINE float rn_mul(float a, float b) { return a * b; }
ND_DEV_INLINE float rn_add(float a, float b) { return a + b; }
ND_DEV_INLINE double rn_mul(double a, double b) { return a * b; }
ND_DEV_INLINE double rn_add(double a, double b) { return a + b; }
ND_DEV_INLINE double fma_d(double a, double b, double c) { return ::fma(a, b, c); }
ND_DEV_INLINE float load_ro(const float* p) { return *p; }
ND_DEV_INLINE int32_t float_bits(float x) {
  int32_t b;
  memcpy(&b, &x, sizeof(b));
  return b;
}
// IEEE binary16 bits of x, rounded to nearest even (host builds of the ray program)
ND_DEV_INLINE uint16_t half_bits(float x) {
  uint32_t u;
  memcpy(&u, &x, sizeof(u));
  const uint32_t sign = (u >> 16) & 0x8000u, ax = u & 0x7fffffffu;
  if (ax >= 0x7f800000u) return uint16_t(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0u));  // inf / NaN
  if (ax >= 0x477ff000u) return uint16_t(sign | 0x7c00u);                                      // overflow
  if (ax < 0x38800000u) {                                                                      // subnormal / 0
    if (ax < 0x33000000u) return uint16_t(sign);
    const uint32_t e = ax >> 23, m = (ax & 0x7fffffu) | 0x800000u;
    const uint32_t shift = 126u - e, q = m >> shift, rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1u);
    return uint16_t(sign | (q + ((rem > half || (rem == half && (q & 1u))) ? 1u : 0u)));
  }
  const uint32_t q = (ax - 0x38000000u) >> 13, rem = ax & 0x1fffu;
  return uint16_t(sign | (q + ((rem > 0x1000u || (rem == 0x1000u && (q & 1u))) ? 1u : 0u)));
}
#endif

constexpr int kMaxIterations = 4096;   // watchdog cap on de_iterations()
constexpr int kShadowMaxSteps = 40;    // SHADOW_MAX_STEPS tpl:2353
constexpr double kShadowBias = 0.004;  // SHADOW_BIAS tpl:2344
constexpr double kShadowHitEps = 0.0005;
constexpr double kShadowMinStep = 0.001;
constexpr double kSimpleAmbient = 0.18;  // SIMPLE_AMBIENT tpl:4418

// Per-view record the kernels read (built on the host from nd_view_desc).
constexpr int kAccelMaxCascades = 8;  // MAX_CASCADES tpl:31, accel.zig:8

struct DevView {
  double org[3];
  double fwd[3];
  double right[3];
  double up[3];
  double uright[3];     // unit right / up for the camera-mounted key light
  double uup[3];
  double light[3];      // unit direction to the light (shadow / Lambert)
  double aspect;
  double footprint;     // hq_footprint_px * 2 / height
  double max_dist;
  int64_t ray_offset;   // first work-item index of this view inside its launch
  int64_t out_offset;   // first G-buffer index of this view
  int64_t rays;
  uint64_t seed;
  float params[ND_MAX_PARAMS];
  nd_trap_desc trap;
  float eps_coef, eps_floor, normal_h_coef, shadow_k, factor;
  int32_t width, height, tile_x, tile_y, tile_w, tile_h, spp;
  int32_t max_steps, refine, verify, hq, normal_mode, shadow, use_light;
  int32_t code;         // formula index inside the kernel's formula set
  int32_t max_samples;  // max_steps * (1 + refine budget) + bisect budget
  int32_t dir64;        // ray directions need FP64 (deep-zoom cameras)
  int32_t user_index;   // the view's index in the caller's array
  int32_t exact_hit;    // bisect for the whole budget (ND_VIEW_EXACT_HIT)
  int32_t scene;        // index into the launch's scene table, -1: the single instance above
  // empty-space accelerator of this view (accel_levels 0: none): cascade l covers
  // accel_res^3 cells of size accel_prm[l][3] from corner accel_prm[l][0..2]
  int32_t accel_levels;
  int32_t accel_res;
  float accel_safety;
  float* accel_grid;    // [level][z][y][x] safe skip distances
  float accel_prm[kAccelMaxCascades][4];
  float accel_inv[kAccelMaxCascades];  // 1 / cell size
  float accel_cam[3];   // the camera position the cascades are centred on (f32)
  float accel_k;        // 1 / ((res / 2 - 1) * finest cell): lookup start level
  ndw::ImageRef image;  // the formula image (texels nullptr: none)
  // n / d for 0 <= n < 2^31 as (n * m) >> s (DivMagic): d = the tile's pixels, d = its width
  uint32_t npix_m, npix_s, width_m, width_s;
};

// Exact unsigned division by a divisor fixed per view, for dividends below 2^31:
// with l = ceil(log2 d), m = ceil(2^(31+l) / d) < 2^32 and s = 31 + l,
// floor(n / d) = (n m) >> s for every 0 <= n < 2^31 (the rounding error of m is
// below d, so n m / 2^s exceeds n / d by less than 2^-l <= 1/d).  A 32-bit division
// by a variable is a long instruction sequence on the GPU; this is one wide multiply
// and a shift.
ND_DEV_INLINE void div_magic(uint32_t d, uint32_t* m, uint32_t* s) {
  uint32_t l = 0;
  while (l < 31 && (uint64_t(1) << l) < d) ++l;
  *s = 31 + l;
  *m = uint32_t(((uint64_t(1) << (31 + l)) + d - 1) / (d ? d : 1));
}
ND_DEV_INLINE uint32_t div_by(uint32_t n, uint32_t m, uint32_t s) { return uint32_t((uint64_t(n) * m) >> s); }

struct Stats {
  unsigned long long rays, de_evals, march_evals, normal_evals, shadow_evals, hits, refills;
  unsigned int timeouts, pad;
};

// One entry of the deferred shade pass's hit list: the launch-local ray index, the DE
// evaluations its march used (the shade pass writes the ray's total once) and the FP64
// hit distance.  The surface pass reads its hits in list order, 16 B each and
// coalesced, instead of fetching each hit's distance from a per-ray array.
struct HitEntry {
  int32_t item;
  uint32_t march_evals;
  double t;
};

// One entry of the shadow queue (the wavefront shadow pass, after cs_wf_shadow
// tpl:5333-5346): a hit whose view casts a shadow ray, with what the surface pass
// computed for it: the shadow ray's origin (hit + normal x SHADOW_BIAS, FP64), the
// unit normal (for the Lambert level once the visibility is known) and the DE
// evaluations the ray has used so far (march + normal taps).
struct ShadowEntry {
  int32_t item;
  uint32_t evals;
  float nx, ny, nz;
  int32_t pad;
  double ox, oy, oz;
};

struct LaunchArgs {
  const DevView* views;       // device
  int32_t nviews;
  int64_t total_rays;
  nd_gbuffer out;             // device pointers
  double* t_hit;              // FP64 hit distance per G-buffer slot (-1 on a miss), for the trap pass
  unsigned long long* counter;  // persistent work counter (zeroed before launch)
  Stats* stats;
  int32_t refill_threshold;
  int32_t chunk;              // rays a warp takes from the work counter at a time
  int32_t accel_chain;        // accelerator jumps per lane and pass (0: no limit)
  int64_t deadline_ns;        // watchdog budget (globaltimer units)
  // Deferred shading: the persistent march ends a hit ray at its hit and appends it
  // to hit_list; the shade pass then evaluates the normal taps coherently.
  struct HitEntry* hit_list;  // hits of the launch (nullptr: shading inline)
  unsigned int* hit_count;    // entries in hit_list (zeroed before launch)
  const struct DevScene* scenes;  // multi-instance scenes of the launch's views (may be null)
  // Wavefront shadow pass: the surface pass appends hits whose view casts a shadow
  // ray to shadow_queue; a persistent shadow kernel then marches them with the same
  // warp-ballot refill as the primary march (nullptr: shadow rays inline).
  ShadowEntry* shadow_queue;
  unsigned int* shadow_count;           // entries in shadow_queue (zeroed before launch)
  unsigned long long* shadow_counter;   // the shadow kernel's work counter (zeroed before launch)
};

// --------------------------------------------------------------- orbit trap
// OrbitTrap accumulator: tpl:1227-1289.
template <class T> struct TrapAcc {
  T x, y, z, w;
};

template <class T> ND_HD_INLINE T trap_distance(const nd_trap_desc& t, ndw::v3<T> z) {
  using ndw::v3;
  const v3<T> q = z - v3<T>(T(t.center[0]), T(t.center[1]), T(t.center[2]));
  switch (t.shape) {
    case ND_TRAP_SPHERE: return ndw::abs(ndw::length(q) - T(t.radius));
    case ND_TRAP_BOX: {
      const v3<T> e = ndw::abs(q) - v3<T>(T(t.box[0]), T(t.box[1]), T(t.box[2]));
      return ndw::abs(ndw::length(ndw::max(e, v3<T>(T(0)))) + ndw::min(ndw::max(e.x, ndw::max(e.y, e.z)), T(0)));
    }
    case ND_TRAP_CROSS: return ndw::min(ndw::abs(q.x), ndw::min(ndw::abs(q.y), ndw::abs(q.z)));
    case ND_TRAP_TORUS: {
      const T a = ndw::sqrt(q.x * q.x + q.z * q.z) - T(t.radius);
      return ndw::abs(ndw::sqrt(a * a + q.y * q.y) - T(t.tube));
    }
    default: return ndw::length(q);
  }
}

template <class T> ND_HD_INLINE TrapAcc<T> trap_begin(const nd_trap_desc& t) {
  const bool high = t.mode != ND_TRAP_MAX && t.mode != ND_TRAP_AVERAGE;
  return TrapAcc<T>{high ? T(1e6) : T(0), T(0), T(0), T(1e6)};
}

template <class T>
ND_HD_INLINE void trap_update(TrapAcc<T>& a, const nd_trap_desc& t, ndw::v3<T> z, bool changed, int it) {
  const T d = trap_distance(t, z);
  a.w = d;
  if (t.mode == ND_TRAP_MAX) {
    a.x = ndw::max(a.x, d);
  } else if (t.mode == ND_TRAP_AVERAGE) {
    if (changed) {
      a.x += d;
      a.y += T(1);
    }
  } else if (t.mode == ND_TRAP_ITERATION) {
    if (d < a.x) {
      a.x = d;
      a.z = T(it);
    }
  } else {
    a.x = ndw::min(a.x, d);
  }
}

template <class T> ND_HD_INLINE T trap_finish(const TrapAcc<T>& a, const nd_trap_desc& t, int iters) {
  if (t.mode == ND_TRAP_AVERAGE) return a.y > T(0.5) ? a.x / ndw::max(a.y, T(1)) : a.w;
  if (t.mode == ND_TRAP_LAST) return a.w;
  if (t.mode == ND_TRAP_ITERATION) return (a.z + T(1)) / T(iters > 1 ? iters : 1);
  return a.x;
}

template <class T> struct DEOut {
  T d;
  T trap;
  int iters;
};

// Parameter access for formula code: p[i] reads the view's packed params.
template <class T> struct ParamRef {
  const float* v;
  const ndw::ImageRef* img = nullptr;  // the view's formula image (image_info)
  ND_HD_INLINE T operator[](int i) const { return T(v[i]); }
  ND_HD_INLINE const ndw::ImageRef* image() const { return img; }
};

// formula_N (fractal_renderer.zig:490-512) + the single-instance scene_de
// (tpl:1611-1626, 1756-1779): identity instance transform, DE scaled by factor.
// With kTrap the orbit trap and the count of iterations that changed the carry
// are accumulated too; the march itself only needs the distance, so the kernels
// evaluate the trap once per hit, at the hit point, in a separate pass.
//
// de_step(carry, pos, p) is a pure function of its arguments (the contract gives it
// no iteration index), so once one iteration returns its input carry unchanged
// every later iteration would too, and the orbit-trap updates they would make
// leave the accumulator as it is (min, max, last and iteration modes see the same
// distance again; average mode only counts changed iterations).  The trap
// evaluation stops right after recording that fixed point (the first unchanged
// carry is still recorded: on the first iteration it is the only record).  The distance-only evaluation of the march
// runs every iteration instead: testing the carry costs more per iteration than the
// iterations it would skip (an escaped Mandelbulb point's step is one length and one
// comparison), and the loop then matches march_to's evaluation exactly.
//
// PR is the parameter accessor (p[i]); the adjoint instantiates the formula code
// with dual numbers for T and a PR whose entries carry tangents.
template <class F, class T, bool kTrap, class PR>
ND_DEV_INLINE DEOut<T> formula_de_p(ndw::v3<T> pos, const PR& p, const nd_trap_desc& trap, float factor) {
  ndw::IterCarry<T> c{pos, T(1)};
  TrapAcc<T> acc;
  if constexpr (kTrap) acc = trap_begin<T>(trap);
  int n = F::template iterations<T, PR>(p);
  n = n < kMaxIterations ? n : kMaxIterations;
  int changed = 0;
  for (int it = 0; it < n; ++it) {
    if constexpr (kTrap) {
      const ndw::v3<T> zp = c.z;
      const T drp = c.dr;
      c = F::template step<T, PR>(c, pos, p);
      const bool ch = (c.z.x != zp.x) | (c.z.y != zp.y) | (c.z.z != zp.z);
      changed += ch ? 1 : 0;
      trap_update(acc, trap, c.z, ch, it);
      // fixed point: every later update would see this same carry (the one just
      // recorded), so nothing changes any more
      if (!ch && !(c.dr != drp)) break;
    } else {
      c = F::template step<T, PR>(c, pos, p);
    }
  }
  DEOut<T> o;
  o.d = F::template finalize<T, PR>(c) * T(factor);
  if constexpr (kTrap) o.trap = trap_finish(acc, trap, n);
  else o.trap = T(0);
  o.iters = changed;
  return o;
}

template <class F, class T, bool kTrap>
ND_DEV_INLINE DEOut<T> formula_de(ndw::v3<T> pos, const float* params, const nd_trap_desc& trap, float factor,
                                  const ndw::ImageRef* image = nullptr) {
  return formula_de_p<F, T, kTrap, ParamRef<T>>(pos, ParamRef<T>{params, image}, trap, factor);
}

// A compile-time list of formulas; code selects one (warp-uniform in practice,
// because batched views are ordered by formula).  de_with evaluates the DE alone
// (no trap) with a caller-supplied parameter accessor.
// eval / step / finalize dispatch on a code like the reference's eval_formula /
// eval_step / eval_finalize (fractal_renderer.zig:529-534); a code outside the set
// gives NO_SURFACE_DE (1e6) / the carry unchanged.
template <class... Fs> struct FormulaSet;
template <class F> struct FormulaSet<F> {
  template <class T, bool kTrap = false>
  static ND_DEV_INLINE DEOut<T> de(int, ndw::v3<T> pos, const DevView& v) {
    return formula_de<F, T, kTrap>(pos, v.params, v.trap, v.factor, &v.image);
  }
  template <class T, class PR>
  static ND_DEV_INLINE DEOut<T> de_with(int, ndw::v3<T> pos, const PR& p, const DevView& v) {
    return formula_de_p<F, T, false, PR>(pos, p, v.trap, v.factor);
  }
  template <class T, bool kTrap>
  static ND_DEV_INLINE DEOut<T> eval(int code, ndw::v3<T> pos, const float* params, const nd_trap_desc& trap) {
    if (code != 0) return DEOut<T>{T(1e6), T(0), 0};
    return formula_de<F, T, kTrap>(pos, params, trap, 1.0f);
  }
  template <class T>
  static ND_DEV_INLINE ndw::IterCarry<T> step(int code, ndw::IterCarry<T> c, ndw::v3<T> pos, const float* params) {
    if (code != 0) return c;
    return F::template step<T, ParamRef<T>>(c, pos, ParamRef<T>{params});
  }
  template <class T> static ND_DEV_INLINE T finalize(int code, ndw::IterCarry<T> c) {
    if (code != 0) return T(1e6);
    return F::template finalize<T, ParamRef<T>>(c);
  }
};
template <class F, class G, class... Rest> struct FormulaSet<F, G, Rest...> {
  template <class T, bool kTrap = false>
  static ND_DEV_INLINE DEOut<T> de(int code, ndw::v3<T> pos, const DevView& v) {
    if (code == 0) return formula_de<F, T, kTrap>(pos, v.params, v.trap, v.factor, &v.image);
    return FormulaSet<G, Rest...>::template de<T, kTrap>(code - 1, pos, v);
  }
  template <class T, class PR>
  static ND_DEV_INLINE DEOut<T> de_with(int code, ndw::v3<T> pos, const PR& p, const DevView& v) {
    if (code == 0) return formula_de_p<F, T, false, PR>(pos, p, v.trap, v.factor);
    return FormulaSet<G, Rest...>::template de_with<T, PR>(code - 1, pos, p, v);
  }
  template <class T, bool kTrap>
  static ND_DEV_INLINE DEOut<T> eval(int code, ndw::v3<T> pos, const float* params, const nd_trap_desc& trap) {
    if (code == 0) return formula_de<F, T, kTrap>(pos, params, trap, 1.0f);
    return FormulaSet<G, Rest...>::template eval<T, kTrap>(code - 1, pos, params, trap);
  }
  template <class T>
  static ND_DEV_INLINE ndw::IterCarry<T> step(int code, ndw::IterCarry<T> c, ndw::v3<T> pos, const float* params) {
    if (code == 0) return F::template step<T, ParamRef<T>>(c, pos, ParamRef<T>{params});
    return FormulaSet<G, Rest...>::template step<T>(code - 1, c, pos, params);
  }
  template <class T> static ND_DEV_INLINE T finalize(int code, ndw::IterCarry<T> c) {
    if (code == 0) return F::template finalize<T, ParamRef<T>>(c);
    return FormulaSet<G, Rest...>::template finalize<T>(code - 1, c);
  }
};

// --------------------------------------------------------------- scenes
// A multi-instance scene as the kernels read it (built on the host from
// nd_scene_desc): per instance the inverse placement and DE factor precomputed.
struct DevInstance {
  float params[ND_MAX_PARAMS];
  float mparams[ND_MAX_MIXINS][ND_MAX_PARAMS];
  float col[3][3];     // rotation frame columns: local_i = (col_i . (p - off)) / s_i
  float off[3];
  float s[3];          // signed scale, |s| >= 0.001 (instance_scale_magnitude)
  float factor;        // min |s| * clamp(step_safety, 0.001, 1)
  float blend_k;
  nd_trap_desc trap;
  int32_t code, hidden, combine, mixin_count, base_n, total_n;
  int32_t mcode[ND_MAX_MIXINS], miters[ND_MAX_MIXINS];
};
struct DevScene {
  int32_t count, carve_count;
  DevInstance inst[ND_MAX_INSTANCES];
  float carves[ND_MAX_CARVES][4];
};

// combine_de (tpl:1708-1730), the distance only.
template <class T> ND_DEV_INLINE T combine_de(int mode, T d, T di, T k) {
  if (mode == ND_COMBINE_UNION) return ndw::min(d, di);
  if (mode == ND_COMBINE_SMOOTH_MIN) return ndw::smin(d, di, k);
  if (mode == ND_COMBINE_SMOOTH_MIX) return ndw::smix(d, di, k);
  if (mode == ND_COMBINE_SMOOTH_MAX) return ndw::smax(d, di, k);
  if (mode == ND_COMBINE_SMOOTH_INV_MAX) return ndw::ssub(di, d, k);
  if (mode == ND_COMBINE_SMOOTH_MIN_LIN) return ndw::smin_lin(d, di, k);
  return ndw::smin_nlin(d, di, k);
}

// The material weight of combine_de (tpl:1708-1730): how much of the scene so far
// (against the new instance) a hit's material keeps; k <= SMOOTH_K_MIN is hard.
template <class T> ND_DEV_INLINE T combine_weight(int mode, T d, T di, T k) {
  const bool hard = k <= T(0.0001);
  const T closer = di < d ? T(0) : T(1);
  if (mode == ND_COMBINE_SMOOTH_MIN || mode == ND_COMBINE_SMOOTH_MIX)
    return hard ? closer : ndw::clamp(T(0.5) + T(0.5) * (di - d) / k, T(0), T(1));
  if (mode == ND_COMBINE_SMOOTH_MAX)
    return hard ? (di > d ? T(0) : T(1)) : ndw::clamp(T(0.5) - T(0.5) * (di - d) / k, T(0), T(1));
  if (mode == ND_COMBINE_SMOOTH_INV_MAX)
    return hard ? (-di > d ? T(0) : T(1)) : T(1) - ndw::clamp(T(0.5) - T(0.5) * (d + di) / k, T(0), T(1));
  return closer;  // union, smooth min-lin / min-nlin
}

// eval_mixed (tpl:1361-1392) with hybrid_cycle_len / hybrid_step (tpl:1335-1359),
// distance before the instance factor; the trap follows every step.
template <class Set, class T, bool kTrap>
ND_DEV_INLINE DEOut<T> eval_mixed(const DevInstance& in, ndw::v3<T> pos) {
  ndw::IterCarry<T> c{pos, T(1)};
  TrapAcc<T> acc;
  if constexpr (kTrap) acc = trap_begin<T>(in.trap);
  const int base_n = in.base_n > 0 ? in.base_n : 0;
  const int mixins = in.mixin_count < ND_MAX_MIXINS ? in.mixin_count : ND_MAX_MIXINS;
  int cycle = base_n;
  for (int j = 0; j < mixins; ++j) cycle += in.miters[j] > 0 ? in.miters[j] : 0;
  if (cycle < 1) cycle = 1;
  int total = in.total_n > 0 ? in.total_n : 0;
  total = total < kMaxIterations ? total : kMaxIterations;
  int changed = 0;
  for (int it = 0; it < total; ++it) {
    int pos_in = it % cycle;
    int code = in.code;
    const float* p = in.params;
    bool have = true;
    if (pos_in >= base_n) {
      pos_in -= base_n;
      have = false;
      for (int j = 0; j < mixins; ++j) {
        const int nj = in.miters[j] > 0 ? in.miters[j] : 0;
        if (pos_in < nj) {
          code = in.mcode[j];
          p = in.mparams[j];
          have = true;
          break;
        }
        pos_in -= nj;
      }
    }
    const ndw::v3<T> zp = c.z;
    if (have) c = Set::template step<T>(code, c, pos, p);
    if constexpr (kTrap) {
      const bool ch = (c.z.x != zp.x) | (c.z.y != zp.y) | (c.z.z != zp.z);
      changed += ch ? 1 : 0;
      trap_update(acc, in.trap, c.z, ch, it);
    }
  }
  DEOut<T> o;
  o.d = Set::template finalize<T>(in.code, c);
  if constexpr (kTrap) o.trap = trap_finish(acc, in.trap, total);
  else o.trap = T(0);
  o.iters = changed;
  return o;
}

// instance_de_trap (tpl:1626-1630): the instance's local DE times its factor.
template <class Set, class T, bool kTrap>
ND_DEV_INLINE DEOut<T> instance_de(const DevInstance& in, ndw::v3<T> pos) {
  const T dx = pos.x - T(in.off[0]), dy = pos.y - T(in.off[1]), dz = pos.z - T(in.off[2]);
  const ndw::v3<T> local = ndw::v3<T>(
      (T(in.col[0][0]) * dx + T(in.col[0][1]) * dy + T(in.col[0][2]) * dz) / T(in.s[0]),
      (T(in.col[1][0]) * dx + T(in.col[1][1]) * dy + T(in.col[1][2]) * dz) / T(in.s[1]),
      (T(in.col[2][0]) * dx + T(in.col[2][1]) * dy + T(in.col[2][2]) * dz) / T(in.s[2]));
  DEOut<T> o = in.mixin_count > 0 ? eval_mixed<Set, T, kTrap>(in, local)
                                  : Set::template eval<T, kTrap>(in.code, local, in.params, in.trap);
  o.d = o.d * T(in.factor);
  return o;
}

// scene_de (tpl:1756-1779) and apply_carves (tpl:1741-1753); no domain warps or
// particles (stubs in the reference's default variant).  With kTrap, the trap and
// iteration count of the visible instance with the smallest DE.
template <class Set, class T, bool kTrap>
ND_DEV_INLINE DEOut<T> scene_de(const DevScene& S, ndw::v3<T> pos, double max_dist) {
  const T empty = T(float(max_dist) * 2.0f + 1.0f);  // empty_scene_de
  T d = empty, best = T(0);
  bool first = true;
  DEOut<T> o;
  o.trap = T(0);
  o.iters = 0;
  const int count = S.count > 1 ? (S.count < ND_MAX_INSTANCES ? S.count : ND_MAX_INSTANCES) : 1;
  for (int i = 0; i < count; ++i) {
    const DevInstance& in = S.inst[i];
    if (in.hidden) continue;
    const DEOut<T> di = instance_de<Set, T, kTrap>(in, pos);
    if constexpr (kTrap) {
      if (first || di.d < best) {
        best = di.d;
        o.trap = di.trap;
        o.iters = di.iters;
      }
    }
    d = first ? di.d : combine_de<T>(in.combine, d, di.d, T(in.blend_k));
    first = false;
  }
  if (first) {
    o.d = empty;
    return o;
  }
  const int carves = S.carve_count < ND_MAX_CARVES ? S.carve_count : ND_MAX_CARVES;
  for (int i = 0; i < carves; ++i) {
    const float* c = S.carves[i];
    const T r = T(c[3]);
    const T len = ndw::length(pos - ndw::v3<T>(T(c[0]), T(c[1]), T(c[2])));
    d = ndw::ssub(len - r, d, T(0.2) * r);  // CARVE_BLEND = 0.2
  }
  o.d = d;
  return o;
}

// The DE a view's rays see: its single instance, or (kernels compiled with kScenes)
// its scene.  Only the scene kernels carry the scene code, so that it costs the
// single-instance march no registers.
template <class Set, class T, bool kTrap = false, bool kScenes = false>
ND_DEV_INLINE DEOut<T> view_de(const DevView& v, ndw::v3<T> pos, const DevScene* scenes) {
  if constexpr (kScenes) {
    if (v.scene >= 0) return scene_de<Set, T, kTrap>(scenes[v.scene], pos, v.max_dist);
  }
  return Set::template de<T, kTrap>(v.code, pos, v);
}

// --------------------------------------------------------------- helpers
ND_DEV_INLINE uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct D3 {
  double x, y, z;
};
ND_DEV_INLINE D3 d3(double x, double y, double z) { return D3{x, y, z}; }
ND_DEV_INLINE D3 fmadd(D3 o, D3 d, double t) {
  return D3{fma_d(d.x, t, o.x), fma_d(d.y, t, o.y), fma_d(d.z, t, o.z)};
}

// Ray direction storage: float for ordinary cameras, double for deep-zoom
// cameras whose neighbouring pixels differ by less than an FP32 ulp.
template <bool kDir64> struct Dir;
template <> struct Dir<false> {
  double x, y, z;  // the f32-rounded direction, held widened
  ND_DEV_INLINE void set(D3 d) { x = double(float(d.x)); y = double(float(d.y)); z = double(float(d.z)); }
  ND_DEV_INLINE D3 get() const { return D3{x, y, z}; }
};
template <> struct Dir<true> {
  double x, y, z;
  ND_DEV_INLINE void set(D3 d) { x = d.x; y = d.y; z = d.z; }
  ND_DEV_INLINE D3 get() const { return D3{x, y, z}; }
};

// eps(t) = coef * t + floor in the DE precision, without FMA contraction
// (march_epsilon tpl:1813-1815).
template <class T> ND_DEV_INLINE double march_eps(const DevView& v, double t) {
  return double(rn_add(rn_mul(v.eps_coef, float(t)), v.eps_floor));
}
template <> ND_DEV_INLINE double march_eps<double>(const DevView& v, double t) {
  return rn_add(rn_mul(double(v.eps_coef), t), double(v.eps_floor));
}

// d < eps(t) for a DE value d: an f32 DE value against the f32 epsilon compares the
// same as their widened doubles, so the FP32 DE path tests in f32 and leaves the
// epsilon's widening to the rarer branches that need it in FP64.
template <class T> ND_DEV_INLINE bool below_eps(const T& d, double dd, const DevView& v, double t) {
  if constexpr (std::is_same<T, float>::value) return d < rn_add(rn_mul(v.eps_coef, float(t)), v.eps_floor);
  else return dd < march_eps<T>(v, t);
}

// accel_skip (tpl:428-447): the safe skip recorded for the finest cascade cell that
// holds p, 0 outside every cascade.  The cascades are nested around the camera, so
// "finest cascade holding p" is found from p's Chebyshev distance m to the camera
// instead of by trying every cascade: cascade l surely holds p when
// m <= (res/2 - 1) cell_l and surely does not when m >= (res/2 + 1) cell_l, which
// leaves cascades ceil(log2(m * accel_k)) - 1 and the one above (one more below for
// the rounding of m * accel_k).  The cell index multiplies by 1 / cell where the
// reference divides: the two differ only within an ulp of a cell boundary, where
// both neighbouring cells' skips are safe to that ulp.
ND_DEV_INLINE float accel_skip(const DevView& v, float px, float py, float pz) {
  const float m = fmaxf(fabsf(px - v.accel_cam[0]), fmaxf(fabsf(py - v.accel_cam[1]), fabsf(pz - v.accel_cam[2])));
  const float x = m * v.accel_k;
  int l = 0;
  if (x > 1.0f) {
    const int32_t b = float_bits(x);  // x > 1: a normal number (or +inf)
    const int e = ((b >> 23) & 0xff) - 127 + ((b & 0x7fffff) != 0 ? 1 : 0);  // ceil(log2 x)
    l = e > 2 ? e - 2 : 0;
  }
  const float rf = float(v.accel_res);
  for (; l < v.accel_levels; ++l) {
    const float inv = v.accel_inv[l];
    const float fx = floorf((px - v.accel_prm[l][0]) * inv);
    const float fy = floorf((py - v.accel_prm[l][1]) * inv);
    const float fz = floorf((pz - v.accel_prm[l][2]) * inv);
    if (!(fx >= 0.0f && fy >= 0.0f && fz >= 0.0f && fx < rf && fy < rf && fz < rf)) continue;
    const int r = v.accel_res;
    return load_ro(v.accel_grid + ((int64_t(l) * r + int(fz)) * r + int(fy)) * r + int(fx));
  }
  return 0.0f;
}

// Primary ray of a work item: cs_wf_generate tpl:5120-5127 / fs_simple tpl:4523-4525
// with the tile transform (fractal_renderer.zig:852-863) folded into frame pixels.
// (ux, uy): the camera-plane coordinates of the ray, direction = fwd + ux right + uy up.
ND_DEV_INLINE void ray_uv(const DevView& v, int64_t local, double* ux, double* uy) {
  const int64_t npix = int64_t(v.tile_w) * v.tile_h;
  int px, py;
  int64_t sample;
  if (local < 0x80000000ll && npix < 0x80000000ll) {
    // 32-bit division by the view's precomputed magic numbers
    const uint32_t s = div_by(uint32_t(local), v.npix_m, v.npix_s);
    const uint32_t pix = uint32_t(local) - s * uint32_t(npix);
    const uint32_t row = div_by(pix, v.width_m, v.width_s);
    sample = s;
    px = v.tile_x + int(pix - row * uint32_t(v.tile_w));
    py = v.tile_y + int(row);
  } else {
    sample = local / npix;
    const int64_t pix = local - sample * npix;
    px = v.tile_x + int(pix % v.tile_w);
    py = v.tile_y + int(pix / v.tile_w);
  }
  double jx = 0.5, jy = 0.5;
  if (v.spp > 1) {
    // keyed by the sample's place in the whole frame (sample, row, column), so that
    // a view cut into tiles draws the same rays as the view itself
    const uint64_t key = (uint64_t(sample) * uint64_t(v.height) + uint64_t(py)) * uint64_t(v.width) + uint64_t(px);
    const uint64_t h = splitmix64(v.seed ^ splitmix64(key));
    jx = double(uint32_t(h) >> 8) * (1.0 / 16777216.0);
    jy = double(uint32_t(h >> 32) >> 8) * (1.0 / 16777216.0);
  }
  const double ndc_x = 2.0 * (double(px) + jx) / double(v.width) - 1.0;
  const double ndc_y = 1.0 - 2.0 * (double(py) + jy) / double(v.height);
  *ux = ndc_x * v.aspect;
  *uy = -ndc_y;
}

ND_DEV_INLINE D3 ray_dir(const DevView& v, int64_t local) {
  double ux, uy;
  ray_uv(v, local, &ux, &uy);
  double x = v.fwd[0] + v.right[0] * ux + v.up[0] * uy;
  double y = v.fwd[1] + v.right[1] * ux + v.up[1] * uy;
  double z = v.fwd[2] + v.right[2] * ux + v.up[2] * uy;
  const double inv = 1.0 / sqrt(x * x + y * y + z * z);
  return D3{x * inv, y * inv, z * inv};
}

template <class T> ND_DEV_INLINE ndw::v3<T> to_t(D3 p) { return ndw::v3<T>(T(p.x), T(p.y), T(p.z)); }

// Tetrahedral tap directions (tetra_gradient tpl:1790-1804).
ND_DEV_INLINE D3 tetra_k(int i) {
  return i == 0 ? d3(1, -1, -1) : i == 1 ? d3(-1, -1, 1) : i == 2 ? d3(-1, 1, -1) : d3(1, 1, 1);
}

// Final per-ray outputs (frag_out tpl:3768-3774; simple_geometry tpl:4492-4507).
struct RayResult {
  double t;
  float nx, ny, nz;
  float shade;
  float shadow;
  uint32_t steps, evals;
  bool hit;
};

// The normal as the reference's RGBA16F target (fr:73-76): four halves, w = hit.
ND_DEV_INLINE void write_normal_half(const nd_gbuffer& g, int64_t r, float nx, float ny, float nz, bool hit) {
  struct alignas(8) H4 {
    uint16_t x, y, z, w;
  };
  reinterpret_cast<H4*>(g.normal_half)[r] = H4{half_bits(nx), half_bits(ny), half_bits(nz), uint16_t(hit ? 0x3c00u : 0u)};
}

// Outputs of the march; t_hit (FP64 t on a hit, -1 on a miss) feeds the trap pass.
ND_DEV_INLINE void write_result(const nd_gbuffer& g, double* t_hit, int64_t r, const RayResult& o) {
  // r is the G-buffer index (view out_offset + ray index inside the view)
  g.depth[r] = o.hit ? float(o.t) : 0.0f;
  if (t_hit) t_hit[r] = o.hit ? o.t : -1.0;
  if (g.normal) {
    struct alignas(16) F4 {
      float x, y, z, w;
    };
    reinterpret_cast<F4*>(g.normal)[r] = F4{o.nx, o.ny, o.nz, o.hit ? 1.0f : 0.0f};
  }
  if (g.normal_half) write_normal_half(g, r, o.nx, o.ny, o.nz, o.hit);
  if (g.steps) g.steps[r] = o.steps;
  if (g.shade) g.shade[r] = o.shade;
  if (g.shadow) g.shadow[r] = o.shadow;
  if (g.depth64) g.depth64[r] = o.hit ? o.t : 0.0;
  if (g.evals) g.evals[r] = o.evals;
  if (!o.hit) {
    if (g.trap) g.trap[r] = 0.0f;
    if (g.iters) g.iters[r] = 0u;
  }
}

// Lambert grey level with the camera-mounted key light of simple_geometry, or the
// view's directional light (times the shadow visibility).
ND_DEV_INLINE float lambert(const DevView& v, D3 dir, double nx, double ny, double nz, float vis) {
  double kx, ky, kz;
  if (v.use_light) {
    kx = v.light[0]; ky = v.light[1]; kz = v.light[2];
  } else {
    kx = rn_add(rn_add(-dir.x, rn_mul(v.uup[0], 0.45)), -rn_mul(v.uright[0], 0.35));
    ky = rn_add(rn_add(-dir.y, rn_mul(v.uup[1], 0.45)), -rn_mul(v.uright[1], 0.35));
    kz = rn_add(rn_add(-dir.z, rn_mul(v.uup[2], 0.45)), -rn_mul(v.uright[2], 0.35));
    const double inv = 1.0 / sqrt(rn_add(rn_add(rn_mul(kx, kx), rn_mul(ky, ky)), rn_mul(kz, kz)));
    kx *= inv; ky *= inv; kz *= inv;
  }
  // explicitly rounded (no FMA contraction), so that every kernel gives the same bits
  const double dot = rn_add(rn_add(rn_mul(nx, kx), rn_mul(ny, ky)), rn_mul(nz, kz));
  const double lam = rn_mul(fmax(dot, 0.0), double(vis));
  return float(rn_add(kSimpleAmbient, rn_mul(1.0 - kSimpleAmbient, lam)));
}

ND_DEV_INLINE int find_view(const DevView* views, int nviews, int64_t item) {
  int lo = 0, hi = nviews - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (views[mid].ray_offset <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// find_view, checking first the view a lane marched last: a warp takes runs of
// consecutive rays, so a new ray is usually in the same view.  The same result as
// find_view (the one non-empty view whose ray range holds item).
ND_DEV_INLINE int find_view_from(const DevView* views, int nviews, int64_t item, int hint) {
  if (hint >= 0 && hint < nviews) {
    const int64_t lo = views[hint].ray_offset;
    if (item >= lo && item - lo < views[hint].rays) return hint;
  }
  return find_view(views, nviews, item);
}

// --------------------------------------------------------------- normals
// estimate_normal (tpl:1783-1804) and the 6-tap central difference, one tap at a
// time: the position of tap k around the hit p, the accumulation of its DE value,
// and the unit normal.  The inline (Lane) and the deferred (shade pass) paths both
// use these, so they produce the same bits.
template <class T> ND_DEV_INLINE D3 normal_tap_pos(const DevView& v, D3 p, double t, int k) {
  if (v.normal_mode == ND_NORMAL_CENTRAL) {
    const double h = v.normal_h_coef > 0.0f ? double(v.normal_h_coef) * t : march_eps<T>(v, t);
    const double s = (k & 1) ? -h : h;
    const int ax = k >> 1;
    return d3(p.x + (ax == 0 ? s : 0.0), p.y + (ax == 1 ? s : 0.0), p.z + (ax == 2 ? s : 0.0));
  }
  return fmadd(p, tetra_k(k), march_eps<T>(v, t));
}

ND_DEV_INLINE void normal_accumulate(const DevView& v, int k, double d, float& gx, float& gy, float& gz) {
  if (v.normal_mode == ND_NORMAL_CENTRAL) {
    const float s = float((k & 1) ? -d : d);
    const int ax = k >> 1;
    if (ax == 0) gx += s;
    else if (ax == 1) gy += s;
    else gz += s;
  } else {
    const D3 kk = tetra_k(k);
    gx += float(kk.x * d);
    gy += float(kk.y * d);
    gz += float(kk.z * d);
  }
}

ND_DEV_INLINE void normal_finish(float& gx, float& gy, float& gz) {
  // explicitly rounded, so that every kernel that inlines this rounds the same way
  const float l = sqrtf(rn_add(rn_add(rn_mul(gx, gx), rn_mul(gy, gy)), rn_mul(gz, gz)));
  const float inv = l > 0.0f ? 1.0f / l : 0.0f;
  gx *= inv;
  gy *= inv;
  gz *= inv;
}

// Normal taps of a view (4 tetrahedral or 6 central-difference evaluations).
ND_DEV_INLINE uint32_t normal_taps(const DevView& v) { return v.normal_mode == ND_NORMAL_CENTRAL ? 6u : 4u; }

// --------------------------------------------------------------- work runs
// A warp's share of the persistent kernel's work list: it takes runs of `chunk`
// consecutive ray indices from a 64-bit global counter (one atomicAdd per claim,
// fetch() returns the counter before the add, the same value on every lane) and
// hands them to its idle lanes.  Every warp may add one more run after the list is
// used up, so the counter ends above the ray total by up to warps x the largest
// claim; it is compared with the total in 64 bits before any narrowing, and only
// indices below the total (< 2^31) become 32-bit ray indices.
struct WarpRuns {
  int32_t next = 0, end = 0;  // taken but not yet started: [next, end)
  bool exhausted = false;     // the counter has passed the total

  ND_DEV_INLINE bool have_work() const { return !exhausted || next < end; }

  // Rays for `nidle` idle lanes.  After the call, idle lane r (by rank) with
  // r < used starts ray first_old + r when r < avail, else base + (r - avail).
  struct Claim {
    int32_t avail, first_old, base, used;
    bool fetched;
    ND_DEV_INLINE int32_t item(int r) const { return r < avail ? first_old + r : base + (r - avail); }
  };
  template <class Fetch> ND_DEV_INLINE Claim claim(int nidle, int chunk, int32_t total, Fetch fetch) {
    Claim c;
    c.avail = end - next;
    c.first_old = next;
    c.base = 0;
    c.fetched = false;
    int32_t nnew = 0;
    if (c.avail < nidle && !exhausted) {
      // enough whole runs to fill every idle lane
      const int take = ((nidle - c.avail + chunk - 1) / chunk) * chunk;
      const uint64_t got = fetch(take);
      c.fetched = true;
      if (got < uint64_t(total)) {
        c.base = int32_t(got);
        nnew = total - c.base < take ? total - c.base : take;
      }
      if (got + uint64_t(take) >= uint64_t(total)) exhausted = true;
    }
    c.used = nidle < c.avail + nnew ? nidle : c.avail + nnew;
    if (c.used <= c.avail) {
      next += c.used;
    } else {
      next = c.base + (c.used - c.avail);
      end = c.base + nnew;
    }
    return c;
  }
};

// --------------------------------------------------------------- the ray program
enum Phase : int { PH_MARCH = 0, PH_NORMAL = 1, PH_SHADOW = 2, PH_DONE = 3 };

// State of one ray in flight.  The fields are shared between the phases: in the
// march a = lo and b = hi (march_to's bracket); in the shadow phase a = the
// distance along the shadow ray and b = the soft-shadow factor res; g holds the
// gradient sum during the normal taps and the unit normal after them; k counts
// bisection refines, normal taps or shadow steps.
template <class T, bool kDir64> struct Lane {
  int32_t item;   // work-item index inside the launch, -1 when idle
  int32_t view;
  int32_t phase;
  Dir<kDir64> dir;
  double t, a, b;
  float gx, gy, gz;
  int32_t i, n, k;
  uint32_t evals;
  uint32_t mev;   // evaluations the march used (set when the march ends)
  bool probing, bisecting, resolved, hit;
  bool lazy;        // outputs wait for flush() (the persistent kernel writes them in batches)
  uint8_t pending;  // outputs not yet written: 1 finish's, 2 finish_march's
  float vis;        // shadow visibility of a pending finish

  ND_DEV_INLINE void start(const DevView& v, int32_t it, int32_t vidx, bool lazy_outputs = false) {
    lazy = lazy_outputs;
    pending = 0;
    item = it;
    view = vidx;
    dir.set(ray_dir(v, int64_t(it) - v.ray_offset));
    phase = PH_MARCH;
    t = a = b = 0.0;
    i = n = k = 0;
    probing = true;
    bisecting = resolved = hit = false;
    evals = 0;
    mev = 0;
    if (v.max_samples <= 0) phase = PH_DONE;  // march_to's loop never runs: a miss
  }

  // Position of this lane's next DE sample.
  ND_DEV_INLINE D3 sample_pos(const DevView& v) const {
    const D3 o = d3(v.org[0], v.org[1], v.org[2]);
    const D3 d = dir.get();
    if (phase == PH_MARCH) return fmadd(o, d, probing ? t : 0.5 * (a + b));
    const D3 p = fmadd(o, d, t);
    if (phase == PH_NORMAL) return normal_tap_pos<T>(v, p, t, k);
    // PH_SHADOW: origin = hit + n * bias, then along the light direction
    const D3 so = fmadd(p, d3(gx, gy, gz), kShadowBias);
    return fmadd(so, d3(v.light[0], v.light[1], v.light[2]), a);
  }

  // The accelerator's jumps before a probe (march_to tpl:1890-1900): while the
  // recorded skip at the probe position exceeds eps(t), advance without a DE
  // evaluation; each jump is a step and a sample of march_to's loop.  May end the
  // ray (a miss).
  // At most `chain` jumps (0: no limit); returns true when the ray may probe now,
  // false when it ended or has more jumps to take (in a later pass).
  ND_DEV_INLINE bool accel_skips(const DevView& v, const nd_gbuffer& g, double* t_hit, int chain) {
    const D3 o = d3(v.org[0], v.org[1], v.org[2]);
    for (int jumps = 0;; ++jumps) {
      const D3 p = fmadd(o, dir.get(), t);
      const double skip = double(accel_skip(v, float(p.x), float(p.y), float(p.z)));
      if (!(skip > march_eps<T>(v, t))) return true;
      if (chain > 0 && jumps >= chain) return false;
      a = t;
      t = t + skip;
      ++i;
      ++n;
      if (t > v.max_dist || i >= v.max_steps || n >= v.max_samples) {
        finish(v, g, t_hit, 1.0f);
        return false;
      }
    }
  }

  ND_DEV_INLINE void finish(const DevView& v, const nd_gbuffer& g, double* t_hit, float visibility) {
    if (!hit) mev = evals;
    phase = PH_DONE;
    if (lazy) {
      pending = 1;
      vis = visibility;
      return;
    }
    write_finish(v, g, t_hit, visibility);
  }

  ND_DEV_INLINE void write_finish(const DevView& v, const nd_gbuffer& g, double* t_hit, float vis) const {
    RayResult r;
    r.hit = hit;
    r.t = t;
    r.steps = hit ? uint32_t(i) : uint32_t(v.max_steps);
    r.evals = evals;
    r.nx = hit ? gx : 0.0f;
    r.ny = hit ? gy : 0.0f;
    r.nz = hit ? gz : 0.0f;
    r.shadow = vis;
    r.shade = hit ? lambert(v, dir.get(), gx, gy, gz, vis) : 0.0f;
    write_result(g, t_hit, v.out_offset + (int64_t(item) - v.ray_offset), r);
  }

  // Write the outputs a lazy lane left pending.
  ND_DEV_INLINE void flush(const DevView& v, const nd_gbuffer& g, double* t_hit) {
    if (pending == 1) write_finish(v, g, t_hit, vis);
    else if (pending == 2) write_march(v, g, t_hit);
    pending = 0;
  }

  // The outputs of a miss (write_finish with hit = false and visibility 1).
  ND_DEV_INLINE void write_miss(const DevView& v, const nd_gbuffer& g, double* t_hit) const {
    RayResult r;
    r.hit = false;
    r.t = t;
    r.steps = uint32_t(v.max_steps);
    r.evals = evals;
    r.nx = r.ny = r.nz = 0.0f;
    r.shadow = 1.0f;
    r.shade = 0.0f;
    write_result(g, t_hit, v.out_offset + (int64_t(item) - v.ray_offset), r);
  }

  // flush for a march that defers all shading (advance<true>): a lane that finished
  // without a hit is a miss, one with a hit waits for the surface pass.
  ND_DEV_INLINE void flush_deferred(const DevView& v, const nd_gbuffer& g, double* t_hit) {
    if (pending == 1) write_miss(v, g, t_hit);
    else if (pending == 2) write_march(v, g, t_hit);
    pending = 0;
  }

  ND_DEV_INLINE void begin_normal(double at) {
    mev = evals;
    t = at;
    hit = true;
    phase = PH_NORMAL;
    k = 0;
    gx = gy = gz = 0.0f;
  }

  // Deferred shading: a hit ends here with the march's outputs (depth, FP64 t,
  // steps, evaluations); the shade pass writes normal, shade and shadow.
  ND_DEV_INLINE void finish_march(const DevView& v, const nd_gbuffer& g, double* t_hit) {
    phase = PH_DONE;
    if (lazy) {
      pending = 2;
      return;
    }
    write_march(v, g, t_hit);
  }

  // (the evaluation count goes to the shade pass with the hit, which writes the total)
  ND_DEV_INLINE void write_march(const DevView& v, const nd_gbuffer& g, double* t_hit) const {
    const int64_t r = v.out_offset + (int64_t(item) - v.ray_offset);
    g.depth[r] = float(t);
    if (t_hit) t_hit[r] = t;
    if (g.steps) g.steps[r] = uint32_t(i);
    if (g.depth64) g.depth64[r] = t;
  }

  template <bool kDeferOnly>
  ND_DEV_INLINE void hit_at(const DevView& v, double at, const nd_gbuffer& g, double* t_hit, bool defer) {
    if constexpr (kDeferOnly) {
      // the ray ends at its hit; the normal and shadow phases are the surface pass's
      t = at;
      hit = true;
      finish_march(v, g, t_hit);
    } else {
      begin_normal(at);
      if (defer) finish_march(v, g, t_hit);
    }
  }

  // Consume one DE result; sets phase = PH_DONE (outputs written) when finished.
  // With defer_shade a hit ends the ray (finish_march) instead of entering PH_NORMAL.
  // kDeferOnly: a march that always defers its shading (every lane is in PH_MARCH or
  // done), compiled without the normal and shadow phases.
  template <bool kDeferOnly = false>
  ND_DEV_INLINE void advance(const DevView& v, const DEOut<T>& de, const nd_gbuffer& g, double* t_hit,
                             bool defer_shade = false) {
    ++evals;
    const double d = double(de.d);
    if (kDeferOnly || phase == PH_MARCH) {
      // one pass of march_to's sample loop (tpl:1881-1960); a = lo, b = hi
      const bool on_hit = v.verify == 0;
      const int refine_budget = on_hit ? 0 : v.refine;
      const int bisect_budget = on_hit ? v.refine : 0;
      const double st = probing ? t : 0.5 * (a + b);
      const bool below = below_eps<T>(de.d, d, v, st);
      ++n;
      if (bisecting) {
        const double e = march_eps<T>(v, st);
        if (below) {
          b = st;
        } else {
          a = st;
        }
        ++k;
        if ((b - a <= e && !v.exact_hit) || k >= bisect_budget) hit_at<kDeferOnly>(v, b, g, t_hit, defer_shade);
        else if (n >= v.max_samples) finish(v, g, t_hit, 1.0f);  // march_to's loop ran out: a miss
        return;
      }
      if (below) {
        if (on_hit && bisect_budget > 0 && (v.exact_hit ? st > a : st - a > march_eps<T>(v, st))) {
          bisecting = true;
          probing = false;
          b = st;
          k = 0;
          if (n >= v.max_samples) finish(v, g, t_hit, 1.0f);
          return;
        }
        hit_at<kDeferOnly>(v, st, g, t_hit, defer_shade);
        return;
      }
      if (probing && on_hit) {
        // a plain sphere-tracing step (no verify refinement): advance by d.  march_to
        // also sets hi, refines and resolved here; with on_hit none of them is read
        // before the bisection's entry sets them again, so the lane leaves them.
        a = t;
        t = t + d;
        ++i;
        if (t > v.max_dist || i >= v.max_steps || n >= v.max_samples) finish(v, g, t_hit, 1.0f);
        return;
      }
      if (probing) {
        a = t;
        b = t + d;
        k = 0;
        resolved = false;
        probing = false;
      } else {
        if (d >= b - st) resolved = true;
        else b = st;
        ++k;
      }
      if (resolved || k >= refine_budget) {
        if (v.hq && !resolved && refine_budget > 0) b = fmin(b, a + fmax(t, 1.0) * v.footprint);
        t = b;
        ++i;
        if (t > v.max_dist || i >= v.max_steps) {
          finish(v, g, t_hit, 1.0f);
          return;
        }
        probing = true;
      }
      if (n >= v.max_samples) finish(v, g, t_hit, 1.0f);
      return;
    }
    if constexpr (kDeferOnly) return;
    if (phase == PH_NORMAL) {
      normal_accumulate(v, k, d, gx, gy, gz);
      ++k;
      if (k < int(normal_taps(v))) return;
      normal_finish(gx, gy, gz);
      const int steps = v.max_steps < kShadowMaxSteps ? v.max_steps : kShadowMaxSteps;
      if (!v.shadow || steps <= 0 || kShadowBias >= 2.0 * v.max_dist) {
        finish(v, g, t_hit, 1.0f);
        return;
      }
      phase = PH_SHADOW;
      a = kShadowBias;  // distance along the shadow ray
      b = 1.0;          // res
      k = 0;
      return;
    }
    // PH_SHADOW: one step of visibility_march (tpl:2294-2341), opaque scene
    if (d < kShadowHitEps) {
      finish(v, g, t_hit, 0.0f);
      return;
    }
    b = fmin(b, double(v.shadow_k) * d / a);
    a += fmax(d, kShadowMinStep);
    ++k;
    const int steps = v.max_steps < kShadowMaxSteps ? v.max_steps : kShadowMaxSteps;
    if (k >= steps || a >= 2.0 * v.max_dist) finish(v, g, t_hit, float(fmin(fmax(b, 0.0), 1.0)));
  }
};

}  // namespace nd

namespace nd {

// The orbit trap and changed-iteration count at a ray's hit point: the formula
// wrapper with its trap (formula_N) evaluated once at org + dir * t_hit.
// p: the hit point, r: the ray's G-buffer slot.
template <class Set, class T, bool kScenes = false>
ND_DEV_INLINE void trap_at_point(const DevView& v, D3 p, int64_t r, const nd_gbuffer& g, const DevScene* scenes) {
  const DEOut<T> de = view_de<Set, T, true, kScenes>(v, to_t<T>(p), scenes);
  if (g.trap) g.trap[r] = float(de.trap);
  if (g.iters) g.iters[r] = uint32_t(de.iters);
}

template <class Set, class T, bool kDir64, bool kScenes = false>
ND_DEV_INLINE void trap_at_hit(const DevView& v, int64_t local, double t, const nd_gbuffer& g,
                               const DevScene* scenes) {
  Dir<kDir64> dir;
  dir.set(ray_dir(v, local));
  const D3 p = fmadd(d3(v.org[0], v.org[1], v.org[2]), dir.get(), t);
  trap_at_point<Set, T, kScenes>(v, p, v.out_offset + local, g, scenes);
}

// The deferred part of a hit ray, in three pieces: surface_at_hit (the normal taps
// at org + dir * t: the same positions, evaluation order and float accumulation as
// the inline PH_NORMAL phase; writes the normal), shadow_visibility (the shadow ray
// when the view has one: the steps of PH_SHADOW) and finish_at_hit (the Lambert
// level, the visibility and the ray's evaluation count).  shade_at_hit chains them;
// with a shadow queue the surface pass queues the shadow ray instead and the shadow
// kernel finishes the ray.

// Does the view cast a shadow ray from its hits? (visibility_march's loop runs)
ND_DEV_INLINE bool casts_shadow(const DevView& v) {
  const int steps = v.max_steps < kShadowMaxSteps ? v.max_steps : kShadowMaxSteps;
  return v.shadow && steps > 0 && kShadowBias < 2.0 * v.max_dist;
}

struct Surface {
  D3 p;              // the hit point
  float gx, gy, gz;  // unit normal
  int taps;
};

template <class Set, class T, bool kDir64, bool kScenes = false>
ND_DEV_INLINE Surface surface_at_hit(const DevView& v, const Dir<kDir64>& dir, double t, int64_t r,
                                     const nd_gbuffer& g, const DevScene* scenes) {
  Surface s;
  s.p = fmadd(d3(v.org[0], v.org[1], v.org[2]), dir.get(), t);
  s.taps = int(normal_taps(v));
  float gx = 0.0f, gy = 0.0f, gz = 0.0f;
  for (int k = 0; k < s.taps; ++k) {
    const DEOut<T> de = view_de<Set, T, false, kScenes>(v, to_t<T>(normal_tap_pos<T>(v, s.p, t, k)), scenes);
    normal_accumulate(v, k, double(de.d), gx, gy, gz);
  }
  normal_finish(gx, gy, gz);
  s.gx = gx;
  s.gy = gy;
  s.gz = gz;
  if (g.normal) {
    struct alignas(16) F4 {
      float x, y, z, w;
    };
    reinterpret_cast<F4*>(g.normal)[r] = F4{gx, gy, gz, 1.0f};
  }
  if (g.normal_half) write_normal_half(g, r, gx, gy, gz, true);
  return s;
}

// The origin of a hit's shadow ray (visibility_march is started at hit + n * bias).
ND_DEV_INLINE D3 shadow_origin(const Surface& s) { return fmadd(s.p, d3(s.gx, s.gy, s.gz), kShadowBias); }

// visibility_march (tpl:2294-2341) toward the light from `so`, opaque scene: the
// visibility, with the DE evaluations in *sev.
template <class Set, class T, bool kScenes = false, bool kAccel = false>
ND_DEV_INLINE float shadow_visibility(const DevView& v, D3 so, const DevScene* scenes, int* sev) {
  float vis = 1.0f;
  int k = 0;
  *sev = 0;
  const int steps = v.max_steps < kShadowMaxSteps ? v.max_steps : kShadowMaxSteps;
  const D3 L = d3(v.light[0], v.light[1], v.light[2]);
  double a = kShadowBias, res = 1.0;
  while (true) {
    const D3 q = fmadd(so, L, a);
    if constexpr (kAccel) {
      // visibility_march tpl:2297-2303: a recorded safe jump instead of an evaluation
      const double skip = double(accel_skip(v, float(q.x), float(q.y), float(q.z)));
      if (skip > kShadowMinStep && double(v.shadow_k) * skip >= res * a) {
        a += skip;
        ++k;
        if (k >= steps || a >= 2.0 * v.max_dist) {
          vis = float(fmin(fmax(res, 0.0), 1.0));
          break;
        }
        continue;
      }
    }
    const DEOut<T> de = view_de<Set, T, false, kScenes>(v, to_t<T>(q), scenes);
    ++*sev;
    const double d = double(de.d);
    if (d < kShadowHitEps) {
      vis = 0.0f;
      break;
    }
    res = fmin(res, double(v.shadow_k) * d / a);
    a += fmax(d, kShadowMinStep);
    ++k;
    if (k >= steps || a >= 2.0 * v.max_dist) {
      vis = float(fmin(fmax(res, 0.0), 1.0));
      break;
    }
  }
  return vis;
}

// The outputs a hit ray's shading ends with.
ND_DEV_INLINE void finish_at_hit(const DevView& v, D3 dir, float gx, float gy, float gz, float vis, uint32_t evals,
                                 int64_t r, const nd_gbuffer& g) {
  if (g.shade) g.shade[r] = lambert(v, dir, gx, gy, gz, vis);
  if (g.shadow) g.shadow[r] = vis;
  if (g.evals) g.evals[r] = evals;
}

// All of it inline: normal, shadow ray, Lambert.  Returns the taps in the low and
// the shadow steps in the high 16 bits.
template <class Set, class T, bool kDir64, bool kScenes = false, bool kAccel = false>
ND_DEV_INLINE uint32_t shade_at_hit(const DevView& v, int64_t local, double t, const nd_gbuffer& g,
                                    const DevScene* scenes, uint32_t march_evals) {
  Dir<kDir64> dir;
  dir.set(ray_dir(v, local));
  const int64_t r = v.out_offset + local;
  const Surface s = surface_at_hit<Set, T, kDir64, kScenes>(v, dir, t, r, g, scenes);
  float vis = 1.0f;
  int sev = 0;
  if (casts_shadow(v)) vis = shadow_visibility<Set, T, kScenes, kAccel>(v, shadow_origin(s), scenes, &sev);
  finish_at_hit(v, dir.get(), s.gx, s.gy, s.gz, vis, march_evals + uint32_t(s.taps + sev), r, g);
  return uint32_t(s.taps) | (uint32_t(sev) << 16);
}

// --------------------------------------------------------------- lite shading
// orbit_trap_to_strip (tpl:2025-2035): the trap value as a position on the colour
// strip (TRAP_MIN_SPAN 1e-4; repeat 1 = fract, 2 = mirror, else clamp).
ND_DEV_INLINE float trap_strip(const nd_trap_desc& t, float v) {
  const float x = v / fmaxf(t.span, 1e-4f) + t.offset;
  if (t.repeat == 1) return x - floorf(x);
  if (t.repeat == 2) {
    const float h = x * 0.5f;
    return 1.0f - fabsf((h - floorf(h)) * 2.0f - 1.0f);
  }
  return fminf(fmaxf(x, 0.0f), 1.0f);
}

struct LiteMaterial {
  float r, g, b, gloss, ior;
};

// sample_gradient (tpl:2003-2023) over stops sorted by position, with mix_material's
// blend of the two neighbours (tpl:1980-2001) for the fields shade_lite reads; no
// stops: default_material (DEFAULT_ALBEDO, DEFAULT_GLOSSINESS, DEFAULT_IOR,
// tpl:1965-1977).
ND_DEV_INLINE LiteMaterial lite_material(const nd_lite_desc& L, float t) {
  const int count = L.color_count < ND_MAX_COLOR_STOPS ? L.color_count : ND_MAX_COLOR_STOPS;
  auto of = [](const nd_color_stop& c) { return LiteMaterial{c.color[0], c.color[1], c.color[2], c.glossiness, c.ior}; };
  if (count <= 0) return LiteMaterial{0.8f, 0.8f, 0.85f, 0.3f, 1.5f};
  if (count == 1 || t <= L.colors[0].position) return of(L.colors[0]);
  if (t >= L.colors[count - 1].position) return of(L.colors[count - 1]);
  for (int i = 0; i < count - 1; ++i) {
    const nd_color_stop& a = L.colors[i];
    const nd_color_stop& b = L.colors[i + 1];
    if (t >= a.position && t <= b.position) {
      const float f = (t - a.position) / fmaxf(b.position - a.position, 1e-4f);  // GRADIENT_MIN_SPAN
      const float h = 1.0f - f;
      auto mx = [h](float x, float y) { return x * (1.0f - h) + y * h; };  // mix(b, a, h)
      return LiteMaterial{mx(b.color[0], a.color[0]), mx(b.color[1], a.color[1]), mx(b.color[2], a.color[2]),
                          mx(b.glossiness, a.glossiness), mx(b.ior, a.ior)};
    }
  }
  return of(L.colors[count - 1]);
}

// hit_material (tpl:2128-2155) of a scene, for the lite pass: every visible
// instance's material (its colour stops at its own trap strip) blended into the
// scene's with combine_de's weight, instance by instance.  colors: the scene's
// ND_MAX_INSTANCES descriptors (only their stops are read).
template <class Set, class T>
ND_DEV_INLINE LiteMaterial scene_lite_material(const DevScene& S, const nd_lite_desc* colors, ndw::v3<T> pos) {
  LiteMaterial m{0.8f, 0.8f, 0.85f, 0.3f, 1.5f};
  T d = T(0);
  bool first = true;
  const int count = S.count > 1 ? (S.count < ND_MAX_INSTANCES ? S.count : ND_MAX_INSTANCES) : 1;
  for (int i = 0; i < count; ++i) {
    const DevInstance& in = S.inst[i];
    if (in.hidden) continue;
    const DEOut<T> di = instance_de<Set, T, true>(in, pos);
    const LiteMaterial mi = lite_material(colors[i], trap_strip(in.trap, float(di.trap)));
    if (first) {
      d = di.d;
      m = mi;
      first = false;
      continue;
    }
    const float h = float(combine_weight<T>(in.combine, d, di.d, T(in.blend_k)));
    auto mx = [h](float b, float a) { return b * (1.0f - h) + a * h; };  // mix_material(m, mi, h)
    m = LiteMaterial{mx(mi.r, m.r), mx(mi.g, m.g), mx(mi.b, m.b), mx(mi.gloss, m.gloss), mx(mi.ior, m.ior)};
    d = combine_de<T>(in.combine, d, di.d, T(in.blend_k));
  }
  return m;
}

// fresnel_schlick (tpl:3424-3430)
ND_DEV_INLINE float fresnel_schlick(float cos_theta, float ior) {
  const float r0root = (1.0f - ior) / (1.0f + ior);
  const float r0 = r0root * r0root;
  const float c = fminf(fmaxf(1.0f - fabsf(cos_theta), 0.0f), 1.0f);
  const float c2 = c * c;
  return r0 + (1.0f - r0) * c2 * c2 * c;
}

// calc_ao (tpl:1817-1840): 5 DE samples along the normal, radius clamp(0.04 t,
// 0.003, 0.25), steps (0.2 + 0.2 i) radius, weights 0.6^i, strength 2.
template <class Set, class T, bool kScenes = false>
ND_DEV_INLINE float calc_ao(const DevView& v, D3 pos, float nx, float ny, float nz, double t, const DevScene* scenes) {
  const float radius = fminf(fmaxf(float(t) * 0.04f, 0.003f), 0.25f);
  float occlusion = 0.0f, weight = 1.0f;
  for (int i = 0; i < 5; ++i) {
    const float step = radius * (0.2f + 0.2f * float(i));
    const D3 q = d3(pos.x + double(nx * step), pos.y + double(ny * step), pos.z + double(nz * step));
    const float d = float(view_de<Set, T, false, kScenes>(v, to_t<T>(q), scenes).d);
    occlusion += fmaxf(step - d, 0.0f) * weight;
    weight *= 0.6f;
  }
  return fminf(fmaxf(1.0f - 2.0f * occlusion / radius, 0.0f), 1.0f);
}

// shade_lite (tpl:4424-4444) at a hit at distance t along the ray with normal n and
// orbit-trap value trap: (1 - F) (albedo (0.15 AO + sum ndotl c) + sum specular),
// AMBIENT_INTENSITY 0.15.  A scene view takes its material from hit_material.
template <class Set, class T, bool kDir64, bool kScenes = false>
ND_DEV_INLINE void lite_at_hit(const DevView& v, const nd_lite_desc& L, int64_t local, double t, float nx, float ny,
                               float nz, float trap, float* rgb, const DevScene* scenes = nullptr,
                               const nd_lite_desc* scene_colors = nullptr) {
  Dir<kDir64> dir;
  dir.set(ray_dir(v, local));
  const D3 dd = dir.get();
  const D3 pos = fmadd(d3(v.org[0], v.org[1], v.org[2]), dd, t);
  LiteMaterial m;
  if constexpr (kScenes) {
    if (v.scene >= 0) m = scene_lite_material<Set, T>(scenes[v.scene], scene_colors + ND_MAX_INSTANCES * v.scene,
                                                      to_t<T>(pos));
    else m = lite_material(L, trap_strip(v.trap, trap));
  } else {
    m = lite_material(L, trap_strip(v.trap, trap));
  }
  const float spec_power = 4.0f + (128.0f - 4.0f) * fminf(fmaxf(m.gloss, 0.0f), 1.0f);  // SPEC_POWER_MIN/MAX
  const float dx = float(dd.x), dy = float(dd.y), dz = float(dd.z);
  const float fresnel = fresnel_schlick(dx * nx + dy * ny + dz * nz, fmaxf(m.ior, 1.0f));
  const float amb = 0.15f * (L.ambient_occlusion ? calc_ao<Set, T, kScenes>(v, pos, nx, ny, nz, t, scenes) : 1.0f);
  float dr = amb, dg = amb, db = amb, sr = 0.0f, sg = 0.0f, sb = 0.0f;
  const int lights = L.light_count < ND_MAX_LIGHTS ? L.light_count : ND_MAX_LIGHTS;
  for (int i = 0; i < lights; ++i) {
    const nd_light& l = L.lights[i];
    float lx, ly, lz, cr = l.color[0] * l.brightness, cg = l.color[1] * l.brightness, cb = l.color[2] * l.brightness;
    if (l.type == ND_LIGHT_POINT) {  // light_sample_ex tpl:2180-2185
      const float tx = l.position_or_direction[0] - float(pos.x), ty = l.position_or_direction[1] - float(pos.y),
                  tz = l.position_or_direction[2] - float(pos.z);
      const float dist = sqrtf(tx * tx + ty * ty + tz * tz);
      const float inv = 1.0f / fmaxf(dist, 1e-4f);  // EPSILON
      lx = tx * inv; ly = ty * inv; lz = tz * inv;
      const float fall = 1.0f / fmaxf(dist * dist, 0.01f);  // LIGHT_MIN_DIST_SQ
      cr *= fall; cg *= fall; cb *= fall;
    } else {  // LIGHT_GLOBAL tpl:2186-2189
      const float px = l.position_or_direction[0], py = l.position_or_direction[1], pz = l.position_or_direction[2];
      const float inv = 1.0f / sqrtf(px * px + py * py + pz * pz);
      lx = px * inv; ly = py * inv; lz = pz * inv;
    }
    const float ndotl = fmaxf(nx * lx + ny * ly + nz * lz, 0.0f);
    if (ndotl <= 0.0f) continue;
    dr += cr * ndotl; dg += cg * ndotl; db += cb * ndotl;
    if (L.specular) {
      float hx = lx - dx, hy = ly - dy, hz = lz - dz;
      const float hl = 1.0f / sqrtf(hx * hx + hy * hy + hz * hz);
      hx *= hl; hy *= hl; hz *= hl;
      const float sp = powf(fmaxf(nx * hx + ny * hy + nz * hz, 0.0f), spec_power) * m.gloss;
      sr += cr * sp; sg += cg * sp; sb += cb * sp;
    }
  }
  const float k = 1.0f - fresnel;
  rgb[0] = k * (m.r * dr + sr);
  rgb[1] = k * (m.g * dg + sg);
  rgb[2] = k * (m.b * db + sb);
}

}  // namespace nd
