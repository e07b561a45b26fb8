// C entry points of the CPU oracle (test infrastructure; see oracle.hpp).
// Built as oracle/_build/liboracle.so by oracle/build_oracle.py; loaded with ctypes
// by the tests and by bench.py's CPU-baseline leg only.
#include <omp.h>
#include <stdint.h>

#include "oracle.hpp"

using namespace oracle;

static void write_ray(const RayOut& o, int64_t i, float* depth, float* normal4, float* trap, uint32_t* steps,
                      uint32_t* iters, float* shade, float* shadow, double* depth64, uint32_t* evals, double* margin) {
  if (depth) depth[i] = float(o.depth);
  if (depth64) depth64[i] = o.depth;
  if (normal4) {
    normal4[4 * i] = float(o.normal[0]);
    normal4[4 * i + 1] = float(o.normal[1]);
    normal4[4 * i + 2] = float(o.normal[2]);
    normal4[4 * i + 3] = o.hit ? 1.0f : 0.0f;
  }
  if (trap) trap[i] = float(o.trap);
  if (steps) steps[i] = o.steps;
  if (iters) iters[i] = o.iters;
  if (shade) shade[i] = float(o.shade);
  if (shadow) shadow[i] = float(o.shadow);
  if (evals) evals[i] = o.evals;
  if (margin) margin[i] = o.margin;
}

// The view's empty-space accelerator grid (when accel_res > 0), built from the DE the
// view's rays see (its formula, or its scene), scaled by de_scale like every DE value.
template <class R>
static bool build_view_accel(AccelGrid& g, const nd_view_desc& v, int kind, const SceneEval<R>* sc, double de_scale,
                             int nthreads) {
  if (v.accel_res <= 0) return false;
  g.place(v.cam_pos, v.max_dist, accel_clamp_levels(v.accel_levels), accel_clamp_res(v.accel_res));
  R p[ND_MAX_PARAMS];
  for (int k = 0; k < ND_MAX_PARAMS; ++k) p[k] = R(v.params[k]);
  const R factor = R(std::min(std::max(double(v.step_safety), 0.001), 1.0));
  g.build(v.accel_safety, nthreads, [&](V3<float> c) {
    const V3<R> q(R(c.x), R(c.y), R(c.z));
    R d = sc ? sc->de(q).d : eval_de<R>(kind, q, p, v.trap, factor).d;
    if (de_scale != 1.0) d = R(double(d) * de_scale);
    return d;
  });
  return true;
}

extern "C" {

// The accelerator grid of one view (its own formula): levels * res^3 floats into
// grid (capacity in floats) and the cascade placement (corner xyz, cell) into prm;
// returns the number of floats, or -1.
int64_t oracle_accel_grid(const nd_view_desc* view, const char* formula_name, int precision, int nthreads,
                          float* grid, int64_t capacity, float* prm) {
  const int kind = formula_index(formula_name);
  if (kind < 0 || view->accel_res <= 0) return -1;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  AccelGrid g;
  if (precision == 32) build_view_accel<float>(g, *view, kind, nullptr, 1.0, nthreads);
  else build_view_accel<double>(g, *view, kind, nullptr, 1.0, nthreads);
  const int64_t n = int64_t(g.v.size());
  if (n > capacity) return -1;
  memcpy(grid, g.v.data(), sizeof(float) * size_t(n));
  for (int l = 0; l < kAccelMaxCascades; ++l)
    for (int a = 0; a < 4; ++a) prm[4 * l + a] = g.prm[l][a];
  return n;
}

int oracle_formula_index(const char* name) { return formula_index(name); }

// The formula image `// @image` formulas read (texels as nd_image_prepare writes them);
// texels NULL clears it.
int oracle_set_image(const uint32_t* texels, int32_t w, int32_t h, const float* slope) {
  OracleImage& im = oracle_image();
  im.texels.clear();
  im.w = im.h = 0;
  for (int k = 0; k < 4; ++k) im.slope[k] = 0.0f;
  if (!texels || w <= 0 || h <= 0) return 0;
  im.texels.assign(texels, texels + size_t(w) * size_t(h) * 4);
  im.w = uint32_t(w);
  im.h = uint32_t(h);
  for (int k = 0; k < 4; ++k) im.slope[k] = slope ? slope[k] : 0.0f;
  return 0;
}

// DE (and trap, changed-iteration count) of a formula at n points, in FP64
// (precision 64) or FP32 (precision 32).
int oracle_de(const char* name, const float* params, const nd_trap_desc* trap, int precision, int64_t n,
              const double* pts, double* de, double* trap_out, int32_t* iters) {
  const int kind = formula_index(name);
  if (kind < 0) return -1;
  nd_trap_desc tz;
  memset(&tz, 0, sizeof(tz));
  const nd_trap_desc& t = trap ? *trap : tz;
  for (int64_t i = 0; i < n; ++i) {
    if (precision == 32) {
      float p[ND_MAX_PARAMS];
      for (int k = 0; k < ND_MAX_PARAMS; ++k) p[k] = params[k];
      const DE<float> r = eval_de<float>(kind, V3<float>(float(pts[3 * i]), float(pts[3 * i + 1]), float(pts[3 * i + 2])), p, t, 1.0f);
      de[i] = r.d;
      if (trap_out) trap_out[i] = r.trap;
      if (iters) iters[i] = r.iters;
    } else {
      double p[ND_MAX_PARAMS];
      for (int k = 0; k < ND_MAX_PARAMS; ++k) p[k] = params[k];
      const DE<double> r = eval_de<double>(kind, V3<double>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), p, t, 1.0);
      de[i] = r.d;
      if (trap_out) trap_out[i] = r.trap;
      if (iters) iters[i] = r.iters;
    }
  }
  return 0;
}

// Trace rays [first, first + n) of one view.  Outputs are indexed 0..n-1; any
// output pointer may be NULL.  nthreads <= 0 uses every core.  de_scale multiplies
// every DE value (1 for the plain march; 1 +- delta probes a ray's stability).
// Returns -1 for an unknown formula name.
int oracle_render(const nd_view_desc* view, const char* formula_name, int precision, int nthreads,
                  int64_t first, int64_t n, float* depth, float* normal4, float* trap, uint32_t* steps,
                  uint32_t* iters, float* shade, float* shadow, double* depth64, uint32_t* evals,
                  double* margin, double de_scale) {
  const int kind = formula_index(formula_name);
  if (kind < 0) return -1;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  AccelGrid grid;
  const bool accel = precision == 32 ? build_view_accel<float>(grid, *view, kind, nullptr, de_scale, nthreads)
                                     : build_view_accel<double>(grid, *view, kind, nullptr, de_scale, nthreads);
#pragma omp parallel num_threads(nthreads)
  {
    Tracer<float> tf(*view, kind);
    Tracer<double> td(*view, kind);
    tf.de_scale = de_scale;
    td.de_scale = de_scale;
    tf.accel = td.accel = accel ? &grid : nullptr;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      const RayOut o = precision == 32 ? tf.trace(first + i) : td.trace(first + i);
      write_ray(o, i, depth, normal4, trap, steps, iters, shade, shadow, depth64, evals, margin);
    }
  }
  return 0;
}

static int scene_kinds(const int32_t* kinds, const int32_t* mixin_kinds, SceneEval<float>& sf, SceneEval<double>& sd) {
  for (int i = 0; i < ND_MAX_INSTANCES; ++i) {
    if (kinds[i] < 0 || kinds[i] >= F_COUNT) return -1;
    sf.kind[i] = sd.kind[i] = kinds[i];
    for (int j = 0; j < ND_MAX_MIXINS; ++j) {
      const int k = mixin_kinds[i * ND_MAX_MIXINS + j];
      if (k < 0 || k >= F_COUNT) return -1;
      sf.mkind[i][j] = sd.mkind[i][j] = k;
    }
  }
  return 0;
}

// The scene DE (and nearest instance's trap and changed-iteration count) at n points.
int oracle_scene_de(const nd_scene_desc* scene, const int32_t* kinds, const int32_t* mixin_kinds, double max_dist,
                    int precision, int64_t n, const double* pts, double* de, double* trap_out, int32_t* iters) {
  SceneEval<float> sf;
  SceneEval<double> sd;
  sf.scene = sd.scene = scene;
  sf.max_dist = sd.max_dist = max_dist;
  if (scene_kinds(kinds, mixin_kinds, sf, sd) != 0) return -1;
  for (int64_t i = 0; i < n; ++i) {
    double d, t;
    int it;
    if (precision == 32) {
      const DE<float> r = sf.de(V3<float>(float(pts[3 * i]), float(pts[3 * i + 1]), float(pts[3 * i + 2])));
      d = r.d; t = r.trap; it = r.iters;
    } else {
      const DE<double> r = sd.de(V3<double>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
      d = r.d; t = r.trap; it = r.iters;
    }
    de[i] = d;
    if (trap_out) trap_out[i] = t;
    if (iters) iters[i] = it;
  }
  return 0;
}

// Trace rays [first, first + n) of one view against a multi-instance scene.  kinds
// holds the oracle formula kind of each instance, mixin_kinds those of each
// instance's mixins (row-major [instance][mixin]).  Outputs as oracle_render.
int oracle_render_scene(const nd_view_desc* view, const nd_scene_desc* scene, const int32_t* kinds,
                        const int32_t* mixin_kinds, int precision, int nthreads, int64_t first, int64_t n,
                        float* depth, float* normal4, float* trap, uint32_t* steps, uint32_t* iters, float* shade,
                        float* shadow, double* depth64, uint32_t* evals, double* margin, double de_scale) {
  SceneEval<float> sf;
  SceneEval<double> sd;
  sf.scene = sd.scene = scene;
  sf.max_dist = sd.max_dist = view->max_dist;
  if (scene_kinds(kinds, mixin_kinds, sf, sd) != 0) return -1;
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  AccelGrid grid;
  const bool accel = precision == 32 ? build_view_accel<float>(grid, *view, kinds[0], &sf, de_scale, nthreads)
                                     : build_view_accel<double>(grid, *view, kinds[0], &sd, de_scale, nthreads);
#pragma omp parallel num_threads(nthreads)
  {
    Tracer<float> tf(*view, kinds[0]);
    Tracer<double> td(*view, kinds[0]);
    tf.de_scale = de_scale;
    td.de_scale = de_scale;
    tf.accel = td.accel = accel ? &grid : nullptr;
    tf.scene = &sf;
    td.scene = &sd;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      const RayOut o = precision == 32 ? tf.trace(first + i) : td.trace(first + i);
      write_ray(o, i, depth, normal4, trap, steps, iters, shade, shadow, depth64, evals, margin);
    }
  }
  return 0;
}

// The primary march alone along given unit directions from the view's camera:
// out4[4 i ..] = hit, t, probe steps, DE evaluations (march_to's MarchResult).
int oracle_march_dirs(const nd_view_desc* view, const char* formula_name, int precision, int64_t n,
                      const double* dirs, double* out4) {
  const int kind = formula_index(formula_name);
  if (kind < 0) return -1;
#pragma omp parallel
  {
    Tracer<float> tf(*view, kind);
    Tracer<double> td(*view, kind);
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      RayOut o;
      memset(&o, 0, sizeof(o));
      const V3<double> d(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]);
      if (precision == 32) {
        DE<float> h{0.0f, 0.0f, 0};
        tf.evals = 0;
        tf.march(d, o, h);
        o.evals = tf.evals;
      } else {
        DE<double> h{0.0, 0.0, 0};
        td.evals = 0;
        td.march(d, o, h);
        o.evals = td.evals;
      }
      out4[4 * i] = o.hit;
      out4[4 * i + 1] = o.depth;
      out4[4 * i + 2] = o.steps;
      out4[4 * i + 3] = o.evals;
    }
  }
  return 0;
}

// Lite shading of rays [first, first + n) of one view from given forward outputs
// (depth64, normal4, trap, indexed 0..n-1): rgba[4 i ..] = rgb, w = hit.
int oracle_shade_lite(const nd_view_desc* view, const char* formula_name, const nd_lite_desc* lite, int precision,
                      int64_t first, int64_t n, const double* depth64, const float* normal4, const float* trap,
                      float* rgba) {
  const int kind = formula_index(formula_name);
  if (kind < 0) return -1;
#pragma omp parallel
  {
    Tracer<float> tf(*view, kind);
    Tracer<double> td(*view, kind);
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      if (!(normal4[4 * i + 3] > 0.5f)) {
        for (int k = 0; k < 3; ++k) rgba[4 * i + k] = lite->background[k];
        rgba[4 * i + 3] = 0.0f;
        continue;
      }
      const V3<double> nn(normal4[4 * i], normal4[4 * i + 1], normal4[4 * i + 2]);
      double rgb[3];
      if (precision == 32) tf.lite(*lite, first + i, depth64[i], nn, trap[i], rgb);
      else td.lite(*lite, first + i, depth64[i], nn, trap[i], rgb);
      for (int k = 0; k < 3; ++k) rgba[4 * i + k] = float(rgb[k]);
      rgba[4 * i + 3] = 1.0f;
    }
  }
  return 0;
}

// Lite shading of a scene view's rays from given forward outputs (as
// oracle_shade_lite); instance_colors: ND_MAX_INSTANCES descriptors of the scene.
int oracle_shade_lite_scene(const nd_view_desc* view, const nd_scene_desc* scene, const int32_t* kinds,
                            const int32_t* mixin_kinds, const nd_lite_desc* lite, const nd_lite_desc* instance_colors,
                            int precision, int64_t first, int64_t n, const double* depth64, const float* normal4,
                            const float* trap, float* rgba) {
  SceneEval<float> sf;
  SceneEval<double> sd;
  sf.scene = sd.scene = scene;
  sf.max_dist = sd.max_dist = view->max_dist;
  if (scene_kinds(kinds, mixin_kinds, sf, sd) != 0) return -1;
#pragma omp parallel
  {
    Tracer<float> tf(*view, kinds[0]);
    Tracer<double> td(*view, kinds[0]);
    tf.scene = &sf;
    td.scene = &sd;
    tf.scene_colors = td.scene_colors = instance_colors;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      if (!(normal4[4 * i + 3] > 0.5f)) {
        for (int k = 0; k < 3; ++k) rgba[4 * i + k] = lite->background[k];
        rgba[4 * i + 3] = 0.0f;
        continue;
      }
      const V3<double> nn(normal4[4 * i], normal4[4 * i + 1], normal4[4 * i + 2]);
      double rgb[3];
      if (precision == 32) tf.lite(*lite, first + i, depth64[i], nn, trap[i], rgb);
      else td.lite(*lite, first + i, depth64[i], nn, trap[i], rgb);
      for (int k = 0; k < 3; ++k) rgba[4 * i + k] = float(rgb[k]);
      rgba[4 * i + 3] = 1.0f;
    }
  }
  return 0;
}

// The oracle's combine_de material weight (f32) at n inputs.
void oracle_combine_weight(int64_t n, const int32_t* mode, const float* d, const float* di, const float* k, float* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = combine_weight<float>(mode[i], d[i], di[i], k[i]);
}

// The oracle's calc_ao at n hit points (positions, normals, t).
int oracle_ao(const nd_view_desc* view, const char* formula_name, int precision, int64_t n, const double* pos,
              const double* nrm, const double* t, double* out) {
  const int kind = formula_index(formula_name);
  if (kind < 0) return -1;
  Tracer<float> tf(*view, kind);
  Tracer<double> td(*view, kind);
  for (int64_t i = 0; i < n; ++i) {
    const V3<double> p(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), q(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
    out[i] = precision == 32 ? tf.ao(p, q, t[i]) : td.ao(p, q, t[i]);
  }
  return 0;
}

// The oracle's orbit_trap_to_strip and fresnel_schlick (f32) at n inputs.
void oracle_strip_fresnel(int64_t n, const float* span_offset_repeat, const float* v, const float* cosv,
                          const float* ior, float* strip, float* fresnel) {
  for (int64_t i = 0; i < n; ++i) {
    const float* s = span_offset_repeat + 3 * i;
    strip[i] = trap_strip<float>(s[0], s[1], int(s[2] + 0.5f), v[i]);
    fresnel[i] = fresnel_schlick<float>(cosv[i], ior[i]);
  }
}

// The oracle's combine (combine_de distance, f32) at n inputs.
void oracle_combine(int64_t n, const int32_t* mode, const float* d, const float* di, const float* k, float* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = combine<float>(mode[i], d[i], di[i], k[i]);
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
