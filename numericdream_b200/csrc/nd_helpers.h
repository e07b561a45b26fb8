// The DE helper library that formula plugins call, plus the orbit trap and the
// per-formula iteration wrapper.  Host and device; templated on the float type T.
//
// Every function here has the behaviour of the WGSL function of the same name in
// NumericDream's shader template (src/gpu/shaders/template.wgsl, line numbers
// below), because formula files call these names and must see the same results.
#pragma once

#include <type_traits>
#include <utility>

#include "nd_wgsl.h"

namespace ndw {

// template.wgsl:57-70 constants used by the helpers
template <class T> ND_HD_INLINE T k_epsilon() { return T(1e-4); }
template <class T> ND_HD_INLINE T k_epsilon_fine() { return T(1e-6); }

// template.wgsl:945-951: reflect each component beyond +-limit back inside.
template <class T> ND_HD_INLINE v3<T> box_fold(v3<T> z, T limit) {
  return clamp(z, v3<T>(-limit), v3<T>(limit)) * T(2) - z;
}

// template.wgsl:953-971: sphere inversion with a floor; radii are squared.
template <class T> ND_HD_INLINE v4<T> sphere_fold(v3<T> z, T dr, T min_radius2, T fixed_radius2) {
#if defined(ND_OPCOUNT_BUILD)
  {
    const T r2 = dot(z, z);
    if (r2 < min_radius2) {
      const T t = fixed_radius2 / min_radius2;
      return v4<T>(z * t, dr * t);
    } else if (r2 < fixed_radius2) {
      const T t = fixed_radius2 / r2;
      return v4<T>(z * t, dr * t);
    }
    return v4<T>(z, dr);
  }
#endif
  // one scale factor instead of three branches (lanes of a warp fall in different
  // shells); outside both radii the factor is 1, and z * 1 == z exactly
  const T r2 = dot(z, z);
  const T q = fixed_radius2 / r2;
  const T t = r2 < min_radius2 ? fixed_radius2 / min_radius2 : (r2 < fixed_radius2 ? q : T(1));
  return v4<T>(z * t, dr * t);
}

// template.wgsl:973-985: inversion in the sphere |d|^2 < radius2 around center.
template <class T> ND_HD_INLINE v4<T> sphere_invert_offset(v3<T> z, T dr, v3<T> center, T radius2) {
#if defined(ND_OPCOUNT_BUILD)
  {
    const v3<T> d = z - center;
    const T r2 = max(dot(d, d), k_epsilon_fine<T>());
    if (r2 < radius2) {
      const T t = radius2 / r2;
      return v4<T>(center + d * t, dr * t);
    }
    return v4<T>(z, dr);
  }
#endif
  // both results computed and selected, so that a warp does not split on the test
  const v3<T> d = z - center;
  const T r2 = max(dot(d, d), k_epsilon_fine<T>());
  const T t = radius2 / r2;
  const bool in = r2 < radius2;
  const v3<T> zi = center + d * t;
  return v4<T>(in ? zi.x : z.x, in ? zi.y : z.y, in ? zi.z : z.z, in ? dr * t : dr);
}

// template.wgsl:987-991: wrap into the cube of side `cell` centred at the origin.
#if defined(__CUDA_ARCH__) && !defined(ND_OPCOUNT_BUILD)
// The FP32 DE on the device: the lattice index k = round(p / cell) comes from adding
// 1.5 * 2^23 in a fused multiply-add, where the float spacing is 1 so the addition
// itself rounds half to even, and subtracting it again.  Two FMA-pipe instructions
// replace the multiply and the FRND of the rounding unit, which the iteration keeps
// busy with its reciprocals.  k is always an integer, so p - k cell is always a lattice
// translate of p; it is the nearest one for |p / cell| < 2^22, and rounds the exact
// product p / cell where the generic form rounds it first.
__device__ __forceinline__ float lattice_index(float x, float inv_cell) {
  const float shift = 12582912.0f;  // 1.5 * 2^23
  return __fadd_rn(__fmaf_rn(x, inv_cell, shift), -shift);
}
#endif
template <class T> ND_HD_INLINE v3<T> lattice_wrap(v3<T> p, T cell) {
#if defined(__CUDA_ARCH__) && !defined(ND_OPCOUNT_BUILD)
  if constexpr (std::is_same<T, float>::value) {
    const float inv = 1.0f / cell;
    return v3<float>(fmaf(-lattice_index(p.x, inv), cell, p.x), fmaf(-lattice_index(p.y, inv), cell, p.y),
                     fmaf(-lattice_index(p.z, inv), cell, p.z));
  }
#endif
  return p - round(p / cell) * cell;
}

// template.wgsl:993-997
template <class T> ND_HD_INLINE T de_finalize_scaled(IterCarry<T> c) { return length(c.z) / abs(c.dr); }
// template.wgsl:999-1003
template <class T> ND_HD_INLINE T de_finalize_plain(IterCarry<T> c) { return length(c.z) / c.dr; }

// template.wgsl:1005-1010: 0.5 log(r) r / dr, capped at r; r and dr floored.
template <class T> ND_HD_INLINE T bulb_log_escape(IterCarry<T> c) {
  const T r = length(c.z);
  const T est = T(0.5) * log(max(r, k_epsilon_fine<T>())) * r / max(c.dr, k_epsilon_fine<T>());
  return min(est, r);
}

// sin and cos of one angle (one shared range reduction for f32/f64).
template <class T> ND_HD_INLINE void sin_cos(T x, T& s, T& c) {
  s = sin(x);
  c = cos(x);
}
ND_HD_INLINE void sin_cos(float x, float& s, float& c) { sincosf(x, &s, &c); }
ND_HD_INLINE void sin_cos(double x, double& s, double& c) { ::sincos(x, &s, &c); }

// template.wgsl:1013 (BULB_BAILOUT) and 1019-1031: one Mandelbulb power step in
// spherical coordinates (theta from +z, phi = atan2(y, x)); no-op once r > 2.
template <class T> ND_HD_INLINE IterCarry<T> bulb_power_step(IterCarry<T> c, v3<T> add, T power) {
  const T r = length(c.z);
  if (r > T(2)) return c;
  const T theta = acos(clamp(c.z.z / r, T(-1), T(1))) * power;
  const T phi = atan2(c.z.y, c.z.x) * power;
  const T rp = pow(r, power - T(1));
  const T zr = rp * r;
  const T dr = rp * power * c.dr + T(1);
  T st, ct, sp, cp;
  sin_cos(theta, st, ct);
  sin_cos(phi, sp, cp);
  const v3<T> z = v3<T>(st * cp, st * sp, ct) * zr + add;
  return IterCarry<T>{z, dr};
}

// template.wgsl:1033-1055: abs then sort components so that x >= y >= z.
template <class T> ND_HD_INLINE v3<T> sort_desc_abs(v3<T> z) {
  v3<T> v = abs(z);
#if defined(__CUDA_ARCH__) && !defined(ND_OPCOUNT_BUILD)
  if constexpr (std::is_same<T, float>::value) {
    // the same three compare-exchanges as a min/max network, so that a warp does not
    // split on them (identical results for non-NaN components: abs gives no -0)
    const float a = fmaxf(v.x, v.y), b = fminf(v.x, v.y);
    const float x = fmaxf(a, v.z), c = fminf(a, v.z);
    return v3<T>(x, fmaxf(b, c), fminf(b, c));
  }
#endif
  if (v.x < v.y) { const T t = v.x; v.x = v.y; v.y = t; }
  if (v.x < v.z) { const T t = v.x; v.x = v.z; v.z = t; }
  if (v.y < v.z) { const T t = v.y; v.y = v.z; v.z = t; }
  return v;
}

// template.wgsl:1057-1077: mirrors across x+y=0, x+z=0, y+z=0 in that order.
template <class T> ND_HD_INLINE v3<T> tetra_fold(v3<T> z) {
  v3<T> v = z;
  if (v.x + v.y < T(0)) { const T t = -v.y; v.y = -v.x; v.x = t; }
  if (v.x + v.z < T(0)) { const T t = -v.z; v.z = -v.x; v.x = t; }
  if (v.y + v.z < T(0)) { const T t = -v.z; v.z = -v.y; v.y = t; }
  return v;
}

// template.wgsl:1079-1083
template <class T> ND_HD_INLINE T wrap_angle(T a, T period) { return a - period * floor(a / period); }

// template.wgsl:1392-1408: right-handed rotations, columns as in the WGSL mat3x3f.
template <class T> ND_HD_INLINE m3<T> rot_x(T a) {
  const T c = cos(a), s = sin(a);
  return m3<T>(v3<T>(T(1), T(0), T(0)), v3<T>(T(0), c, s), v3<T>(T(0), -s, c));
}
template <class T> ND_HD_INLINE m3<T> rot_y(T a) {
  const T c = cos(a), s = sin(a);
  return m3<T>(v3<T>(c, T(0), -s), v3<T>(T(0), T(1), T(0)), v3<T>(s, T(0), c));
}
template <class T> ND_HD_INLINE m3<T> rot_z(T a) {
  const T c = cos(a), s = sin(a);
  return m3<T>(v3<T>(c, s, T(0)), v3<T>(-s, c, T(0)), v3<T>(T(0), T(0), T(1)));
}

// template.wgsl:1085-1093: rot_z * (rot_y * (rot_x * z)) with angles in degrees;
// identity when all three angles are exactly zero.
template <class T> ND_HD_INLINE v3<T> rotate_xyz_deg(v3<T> z, v3<T> deg) {
  if (deg.x == T(0) && deg.y == T(0) && deg.z == T(0)) return z;
  const v3<T> a = radians(deg);
  return mul(rot_z(a.z), mul(rot_y(a.y), mul(rot_x(a.x), z)));
}

// template.wgsl:1095-1098
template <class T> ND_HD_INLINE int32_t primitive_de_iterations() { return 1; }

// template.wgsl:1100-1109: rescale z by 1/size and 1/|dr|; dr becomes 1/size.
template <class T> ND_HD_INLINE IterCarry<T> primitive_de_step(IterCarry<T> c, T size) {
  const T unit_dr = T(1) / max(size, k_epsilon<T>());
  const T f = unit_dr / max(abs(c.dr), k_epsilon_fine<T>());
  return IterCarry<T>{c.z * f, unit_dr};
}

// template.wgsl:1648-1706: smooth combine family; k <= 1e-4 is the hard operation.
template <class T> ND_HD_INLINE T smin(T a, T b, T k) {
  if (k <= T(0.0001)) return min(a, b);
  const T h = clamp(T(0.5) + T(0.5) * (b - a) / k, T(0), T(1));
  return mix(b, a, h) - k * h * (T(1) - h);
}
template <class T> ND_HD_INLINE T smax(T a, T b, T k) {
  if (k <= T(0.0001)) return max(a, b);
  const T h = clamp(T(0.5) - T(0.5) * (b - a) / k, T(0), T(1));
  return mix(b, a, h) + k * h * (T(1) - h);
}
template <class T> ND_HD_INLINE T ssub(T cut, T base, T k) {
  if (k <= T(0.0001)) return max(-cut, base);
  const T h = clamp(T(0.5) - T(0.5) * (base + cut) / k, T(0), T(1));
  return mix(base, -cut, h) + k * h * (T(1) - h);
}
template <class T> ND_HD_INLINE T smin_lin(T a, T b, T k) {
  if (k <= T(0.0001)) return min(a, b);
  return min(b - max(k - a, T(0)), a - max(k - b, T(0)));
}
template <class T> ND_HD_INLINE T smin_nlin(T a, T b, T k) {
  if (k <= T(0.0001)) return min(a, b);
  const T ra = max(k - a, T(0));
  const T rb = max(k - b, T(0));
  return min(b - ra * (k - rb) / k, a - rb * (k - ra) / k);
}
template <class T> ND_HD_INLINE T smix(T a, T b, T k) {
  if (k <= T(0.0001)) return min(a, b);
  const T h = clamp(T(0.5) + T(0.5) * (b - a) / k, T(0), T(1));
  return mix(b, a, h);
}

// ------------------------------------------------------------------ formula images
// The image a formula declares with `// @image` and reads through image_info() and
// image_sample() (template.wgsl:1111-1191).  The texels are prepared on the host by
// nd_image_prepare, four 32-bit words per texel (IMAGE_TEXEL_WORDS): red and green as
// u16 in word 0, blue and alpha in word 1 (R, G, B premultiplied by alpha, then alpha,
// each in [0, 1]), and in words 2 and 3 the per-channel bounds on the change per texel
// within IMAGE_SLOPE_RADIUS_NEAR and _FAR texels as u8 codes (image_slope_decode).
// The reference finds a formula's image through a slot index into one shared buffer;
// here a view carries a pointer to its image, and the formula's parameter accessor
// carries it to image_info().
struct ImageRef {
  const uint32_t* texels;  // nullptr: no image (image_info reports size 0)
  uint32_t width, height;
  float slope[4];          // per channel: the largest change between neighbouring texels
};

template <class T> struct ImageInfo {  // ImageInfo, tpl:1142-1146
  uint32_t base;                       // 0: the texels pointer replaces the shared buffer's offset
  v2<uint32_t> size;
  v4<T> slope;
  const uint32_t* texels;
};
template <class T> struct ImageSample {  // ImageSample, tpl:1158-1162
  v4<T> value;
  v4<T> near;
  v4<T> far;
};

// The accessor's image when it has one (ParamRef of a view in a kernel); the host
// builds of the formula code (op counting) and the dual-number accessor of the adjoint
// see no image.
template <class P, class = void> struct HasImage {
  static constexpr bool value = false;
};
template <class P> struct HasImage<P, decltype(void(std::declval<const P&>().image()))> {
  static constexpr bool value = true;
};
template <class P> ND_HD_INLINE const ImageRef* image_of(const P& p) {
#if defined(__CUDA_ARCH__)
  if constexpr (HasImage<P>::value) return p.image();
#endif
  (void)p;
  return nullptr;
}

ND_HD_INLINE uint32_t image_word(const uint32_t* w, uint32_t i) {
#if defined(__CUDA_ARCH__)
  return __ldg(w + i);
#else
  return w[i];
#endif
}

// image_info (tpl:1148-1155)
template <class T, class P> ND_HD_INLINE ImageInfo<T> image_info(const P& p) {
  const ImageRef* im = image_of(p);
  if (!im || !im->texels) return ImageInfo<T>{0u, v2<uint32_t>(0u, 0u), v4<T>(T(0)), nullptr};
  return ImageInfo<T>{0u, v2<uint32_t>(im->width, im->height),
                      v4<T>(T(im->slope[0]), T(im->slope[1]), T(im->slope[2]), T(im->slope[3])), im->texels};
}

// image_slope_decode (tpl:1164-1168): code c in 1..255 is the bound 2^((c - 255) / 16 + 1),
// 0 is no change.
template <class T> ND_HD_INLINE v4<T> image_slope_decode(uint32_t packed) {
  const T c[4] = {T(packed & 0xffu), T((packed >> 8) & 0xffu), T((packed >> 16) & 0xffu), T(packed >> 24)};
  v4<T> out;
  for (int k = 0; k < 4; ++k) {
    const T s = exp2((c[k] - T(255.0)) / T(16.0) + T(1.0));
    out[k] = c[k] == T(0) ? T(0) : s;
  }
  return out;
}

// image_texel (tpl:1170-1176)
template <class T> ND_HD_INLINE ImageSample<T> image_texel(const ImageInfo<T>& info, uint32_t x, uint32_t y) {
  const uint32_t i = info.base + (y * info.size.x + x) * 4u;
  const uint32_t rg = image_word(info.texels, i), ba = image_word(info.texels, i + 1u);
  const T scale = T(1.0f / 65535.0f);  // IMAGE_U16_SCALE, an f32 constant
  const v4<T> value = v4<T>(T(rg & 0xffffu), T(rg >> 16), T(ba & 0xffffu), T(ba >> 16)) * scale;
  return ImageSample<T>{value, image_slope_decode<T>(image_word(info.texels, i + 2u)),
                        image_slope_decode<T>(image_word(info.texels, i + 3u))};
}

// image_mix (tpl:1178-1180): mix of every field with one weight
template <class T> ND_HD_INLINE ImageSample<T> image_mix(const ImageSample<T>& a, const ImageSample<T>& b, T t) {
  const v4<T> w(t);
  return ImageSample<T>{mix(a.value, b.value, w), mix(a.near, b.near, w), mix(a.far, b.far, w)};
}

// image_sample (tpl:1182-1191): bilinear at uv in [0, 1]^2, clamped at the edges;
// zeros without an image.
template <class T> ND_HD_INLINE ImageSample<T> image_sample(const ImageInfo<T>& info, v2<T> uv) {
  if (info.size.x == 0u || info.size.y == 0u || !info.texels)
    return ImageSample<T>{v4<T>(T(0)), v4<T>(T(0)), v4<T>(T(0))};
  const v2<uint32_t> last = v2<uint32_t>(info.size.x - 1u, info.size.y - 1u);
  const T tx = clamp(uv.x * T(info.size.x) - T(0.5), T(0), T(last.x));
  const T ty = clamp(uv.y * T(info.size.y) - T(0.5), T(0), T(last.y));
  const uint32_t x0 = min(to_u32(tx), last.x), y0 = min(to_u32(ty), last.y);
  const uint32_t x1 = min(x0 + 1u, last.x), y1 = min(y0 + 1u, last.y);
  const T fx = tx - T(x0), fy = ty - T(y0);
  const ImageSample<T> top = image_mix(image_texel(info, x0, y0), image_texel(info, x1, y0), fx);
  const ImageSample<T> bottom = image_mix(image_texel(info, x0, y1), image_texel(info, x1, y1), fx);
  return image_mix(top, bottom, fy);
}

}  // namespace ndw
