// Host-side construction of the kernels' per-view record from nd_view_desc.
#pragma once

#include <math.h>
#include <string.h>

#include <algorithm>

#include "nd_rayprog.h"

namespace nd {

inline DevView make_dev_view(const nd_view_desc& v, int64_t ray_offset, int64_t out_offset, int code) {
  DevView d;
  memset(&d, 0, sizeof(d));
  auto unit = [](const double* a, double* out) {
    const double n = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int i = 0; i < 3; ++i) out[i] = n > 0 ? a[i] / n : 0.0;
  };
  for (int i = 0; i < 3; ++i) {
    d.org[i] = v.cam_pos[i];
    d.fwd[i] = v.fwd[i];
    d.right[i] = v.right[i];
    d.up[i] = v.up[i];
  }
  unit(v.right, d.uright);
  unit(v.up, d.uup);
  const double l[3] = {v.light_dir[0], v.light_dir[1], v.light_dir[2]};
  unit(l, d.light);
  d.use_light = (v.shadow || (l[0] * l[0] + l[1] * l[1] + l[2] * l[2]) > 0) ? 1 : 0;
  d.aspect = double(v.width) / double(v.height);
  d.footprint = double(v.hq_footprint_px) * 2.0 / std::max(double(v.height), 1.0);
  d.max_dist = v.max_dist;
  d.ray_offset = ray_offset;
  d.out_offset = out_offset;
  d.rays = int64_t(v.spp) * v.tile_w * v.tile_h;
  d.seed = v.seed;
  memcpy(d.params, v.params, sizeof(d.params));
  d.trap = v.trap;
  d.eps_coef = v.eps_coef;
  d.eps_floor = v.eps_floor;
  d.normal_h_coef = v.normal_h_coef;
  d.shadow_k = v.shadow_k;
  d.factor = std::min(std::max(v.step_safety, 0.001f), 1.0f);
  d.width = v.width;
  d.height = v.height;
  d.tile_x = v.tile_x;
  d.tile_y = v.tile_y;
  d.tile_w = v.tile_w;
  d.tile_h = v.tile_h;
  d.spp = v.spp;
  d.max_steps = v.max_steps;
  d.refine = v.refine_budget;
  d.verify = v.march_verify;
  d.hq = v.high_quality;
  d.normal_mode = v.normal_mode;
  d.shadow = v.shadow;
  d.code = code;
  d.user_index = 0;
  d.exact_hit = (v.flags & ND_VIEW_EXACT_HIT) != 0 ? 1 : 0;
  d.scene = -1;
  const int refine = v.march_verify ? v.refine_budget : 0;
  const int bisect = v.march_verify ? 0 : v.refine_budget;
  const int64_t ms = int64_t(v.max_steps) * (1 + refine) + bisect;
  d.max_samples = int32_t(std::min<int64_t>(ms, 0x7fffffff));
  // FP64 ray directions when the camera's pixel footprint approaches an FP32 ulp
  // (deep zoom) or when the view asks for them
  const double rn = sqrt(v.right[0] * v.right[0] + v.right[1] * v.right[1] + v.right[2] * v.right[2]);
  const double un = sqrt(v.up[0] * v.up[0] + v.up[1] * v.up[1] + v.up[2] * v.up[2]);
  d.dir64 = ((v.flags & ND_VIEW_DIR64) != 0 || std::max(rn, un) < 1e-3) ? 1 : 0;
  d.image.texels = v.image_texels;
  d.image.width = v.image_texels ? uint32_t(v.image_width) : 0u;
  d.image.height = v.image_texels ? uint32_t(v.image_height) : 0u;
  for (int i = 0; i < 4; ++i) d.image.slope[i] = v.image_slope[i];
  // ray_uv's 32-bit path divides by the tile's pixel count and width (both < 2^31 there)
  const int64_t npix = int64_t(v.tile_w) * v.tile_h;
  div_magic(uint32_t(npix > 0 && npix < 0x80000000ll ? npix : 1), &d.npix_m, &d.npix_s);
  div_magic(uint32_t(v.tile_w > 0 ? v.tile_w : 1), &d.width_m, &d.width_s);
  return d;
}

// Accelerator geometry of a view: resolution clamped to 16..160 and rounded down to a
// multiple of 4 (clampResolution, src/gpu/accel.zig:28-31), 1..8 cascades; 0 = off.
inline int accel_res_of(const nd_view_desc& v) {
  return v.accel_res <= 0 ? 0 : std::min(std::max(v.accel_res, 16), 160) / 4 * 4;
}
inline int accel_levels_of(const nd_view_desc& v) {
  return std::min(std::max(v.accel_levels, 1), kAccelMaxCascades);
}
inline int64_t accel_voxels_of(const nd_view_desc& v) {
  const int64_t r = accel_res_of(v);
  return r ? int64_t(accel_levels_of(v)) * r * r * r : 0;
}

// Cascades centred on the camera (placeCascades, src/gpu/accel.zig:32-56, f32 like
// the reference): the coarsest cell spans 2 max_dist / res, each finer cascade halves
// it, corners snapped to the cascade's cell grid.  grid: levels * res^3 floats.
inline void place_accel(DevView& d, const nd_view_desc& v, float* grid) {
  const int res = accel_res_of(v), levels = accel_levels_of(v);
  d.accel_res = res;
  d.accel_levels = res ? levels : 0;
  d.accel_safety = v.accel_safety;
  d.accel_grid = grid;
  if (!res) return;
  const float res_f = float(res);
  const float coarsest = std::max(2.0f * v.max_dist / res_f, 1e-6f);
  for (int l = 0; l < levels; ++l) {
    const float cell = coarsest / float(1u << (levels - 1 - l));
    const float half = 0.5f * res_f * cell;
    for (int a = 0; a < 3; ++a) d.accel_prm[l][a] = std::floor((float(v.cam_pos[a]) - half) / cell) * cell;
    d.accel_prm[l][3] = cell;
    d.accel_inv[l] = 1.0f / cell;
  }
  for (int a = 0; a < 3; ++a) d.accel_cam[a] = float(v.cam_pos[a]);
  d.accel_k = 1.0f / ((0.5f * res_f - 1.0f) * d.accel_prm[0][3]);
}

// One scene instance as the kernels read it.  code / mcode: the instance's and its
// mixins' formula indices inside the launch's formula set.
inline DevInstance make_dev_instance(const nd_instance_desc& in, int code, const int* mcode) {
  DevInstance d;
  memset(&d, 0, sizeof(d));
  for (int k = 0; k < ND_MAX_PARAMS; ++k) d.params[k] = in.params[k];
  for (int j = 0; j < ND_MAX_MIXINS; ++j) {
    for (int k = 0; k < ND_MAX_PARAMS; ++k) d.mparams[j][k] = in.mixins[j].params[k];
    d.mcode[j] = mcode[j];
    d.miters[j] = in.mixins[j].iterations;
  }
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) d.col[c][r] = in.frame[3 * c + r];
  float mag_min = 1e30f;
  for (int i = 0; i < 3; ++i) {
    d.off[i] = in.offset[i];
    const float mag = std::max(fabsf(in.scale[i]), 0.001f);  // MIN_INSTANCE_SCALE
    d.s[i] = in.scale[i] < 0.0f ? -mag : mag;
    mag_min = std::min(mag_min, mag);
  }
  d.factor = mag_min * std::min(std::max(in.step_safety, 0.001f), 1.0f);
  d.blend_k = in.blend_k;
  d.trap = in.trap;
  d.code = code;
  d.hidden = in.hidden ? 1 : 0;
  d.combine = in.combine_mode;
  d.mixin_count = std::min(std::max(in.mixin_count, 0), ND_MAX_MIXINS);
  d.base_n = in.hybrid_base_iters;
  d.total_n = in.hybrid_total_iters;
  return d;
}

}  // namespace nd
