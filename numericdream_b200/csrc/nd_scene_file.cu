// Scene files (.dream, JSON, version <= 12; src/app/scene_file.zig) read into the
// library's descriptors: the camera, march settings and fractal instances that the
// forward pass uses, as the reference's bench export sets them up (bench.zig:124-155
// with export_image.buildUniforms :97-165: render_settings' max_steps / max_dist /
// precision, high_quality on).  Lights, fog, sky, materials, warps and particles are
// not part of this pass and are ignored.  Host code only.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <utility>
#include <vector>

#include "nd_json.h"
#include "nd_registry.h"

namespace {

using nd_json::JsonParser;
using nd_json::JVal;

// ---------------------------------------------------------------- scene fields
struct Loader {
  std::string err;

  bool fail(const std::string& what) {
    err = what;
    return false;
  }
  static double num(const JVal* v, double dflt) { return v && v->kind == JVal::NUM ? v->num : dflt; }
  static bool boolean(const JVal* v, bool dflt) { return v && v->kind == JVal::BOOL ? v->b : dflt; }
  bool vec3(const JVal* v, const char* what, double out[3]) {
    if (!v || v->kind != JVal::OBJ) return fail(std::string(what) + ": expected {x, y, z}");
    const char* k[3] = {"x", "y", "z"};
    for (int a = 0; a < 3; ++a) {
      const JVal* c = v->get(k[a]);
      if (!c || c->kind != JVal::NUM) return fail(std::string(what) + ": missing " + k[a]);
      out[a] = c->num;
    }
    return true;
  }
  static void vec3_or(const JVal* v, const double dflt[3], float out[3]) {
    double d[3] = {dflt[0], dflt[1], dflt[2]};
    if (v && v->kind == JVal::OBJ) {
      const char* k[3] = {"x", "y", "z"};
      for (int a = 0; a < 3; ++a) d[a] = num(v->get(k[a]), d[a]);
    }
    for (int a = 0; a < 3; ++a) out[a] = float(d[a]);
  }
  // enum tag names as std.json writes them (scene_state.zig)
  bool tag(const JVal* v, const char* const* names, int n, int dflt, const char* what, int32_t* out) {
    if (!v) {
      *out = dflt;
      return true;
    }
    if (v->kind != JVal::STR) return fail(std::string(what) + ": expected a name");
    for (int i = 0; i < n; ++i)
      if (v->str == names[i]) {
        *out = i;
        return true;
      }
    return fail(std::string(what) + ": unknown value \"" + v->str + "\"");
  }

  // FormulaDto {path, params: [{name, value}]}: the formula by its file stem (an
  // empty path is the built-in Mandelbulb, src/gpu/shaders/mandelbrot.wgsl), its
  // @param defaults, then the saved values by name (applyParamDtosTo :484-495),
  // packed in declaration order (packParams, formula.zig:104-108).
  bool formula(const JVal* f, const char* what, int32_t* id, float params[ND_MAX_PARAMS]) {
    if (!f || f->kind != JVal::OBJ) return fail(std::string(what) + ": expected a formula object");
    const JVal* p = f->get("path");
    std::string stem = p && p->kind == JVal::STR ? p->str : std::string();
    const size_t slash = stem.find_last_of("/\\");
    if (slash != std::string::npos) stem = stem.substr(slash + 1);
    if (stem.size() > 5 && stem.compare(stem.size() - 5, 5, ".wgsl") == 0) stem.resize(stem.size() - 5);
    if (stem.empty()) stem = "mandelbrot";
    *id = -1;
    for (int i = 0; i < nd_formula_total(); ++i)
      if (stem == nd_formula_at(i)->name) *id = i;
    if (*id < 0) return fail(std::string(what) + ": formula \"" + stem + "\" is not in this build");
    const nd::FormulaEntry& e = (*nd_formula_at(*id));
    for (int k = 0; k < ND_MAX_PARAMS; ++k) params[k] = k < e.nparams ? e.params[k].default_value : 0.0f;
    const JVal* saved = f->get("params");
    if (saved && saved->kind == JVal::ARR)
      for (const JVal& sp : saved->arr) {
        const JVal* name = sp.get("name");
        const JVal* value = sp.get("value");
        if (!name || name->kind != JVal::STR || !value || value->kind != JVal::NUM) continue;
        for (int k = 0; k < e.nparams; ++k)
          if (name->str == e.params[k].name) {
            params[k] = float(value->num);
            break;
          }
      }
    return true;
  }

  bool trap(const JVal* t, nd_trap_desc* out) {
    static const char* const shapes[] = {"point", "sphere", "box", "cross", "torus"};
    static const char* const modes[] = {"min", "max", "average", "last", "iteration"};
    static const char* const repeats[] = {"clamp", "repeat", "mirror"};
    memset(out, 0, sizeof(*out));
    const double zero[3] = {0, 0, 0}, one[3] = {1, 1, 1};
    const JVal* none = nullptr;
    const JVal* src = t && t->kind == JVal::OBJ ? t : none;
    auto g = [&](const char* k) { return src ? src->get(k) : nullptr; };
    if (!tag(g("shape"), shapes, 5, 0, "trap.shape", &out->shape)) return false;
    if (!tag(g("mode"), modes, 5, 0, "trap.mode", &out->mode)) return false;
    if (!tag(g("repeat"), repeats, 3, 0, "trap.repeat", &out->repeat)) return false;
    vec3_or(g("center"), zero, out->center);
    vec3_or(g("box"), one, out->box);
    out->radius = float(num(g("radius"), 1.0));
    out->tube = float(num(g("tube"), 0.0));
    out->span = float(num(g("span"), 1.5));
    out->offset = float(num(g("offset"), 0.0));
    return true;
  }

  // InstanceDto -> nd_instance_desc (FractalInstanceState.toGpu, scene_state.zig:278-324)
  bool instance(const JVal* in, int idx, nd_instance_desc* out) {
    char what[32];
    snprintf(what, sizeof(what), "instances[%d]", idx);
    if (!in || in->kind != JVal::OBJ) return fail(std::string(what) + ": expected an object");
    memset(out, 0, sizeof(*out));
    if (!formula(in->get("formula"), what, &out->formula, out->params)) return false;
    const double zero[3] = {0, 0, 0}, one[3] = {1, 1, 1};
    vec3_or(in->get("offset"), zero, out->offset);
    float scale[3], rot[3];
    vec3_or(in->get("scale"), one, scale);
    vec3_or(in->get("rotation"), zero, rot);
    const float su = float(num(in->get("scale_uniform"), 1.0));
    for (int a = 0; a < 3; ++a) out->scale[a] = scale[a] * su;
    // eulerFrame (camera.zig:40-60): the columns of Rz * Ry * Rx, angles in radians
    const float k = 3.14159265358979323846f / 180.0f;
    const float rx = rot[0] * k, ry = rot[1] * k, rz = rot[2] * k;
    const float cx = cosf(rx), sx = sinf(rx), cy = cosf(ry), sy = sinf(ry), cz = cosf(rz), sz = sinf(rz);
    const float cols[9] = {cy * cz, cy * sz, -sy,
                           sx * sy * cz - cx * sz, sx * sy * sz + cx * cz, sx * cy,
                           cx * sy * cz + sx * sz, cx * sy * sz - sx * cz, cx * cy};
    memcpy(out->frame, cols, sizeof(cols));
    out->step_safety = float(num(in->get("step_safety"), 1.0));
    out->blend_k = float(num(in->get("blend_k"), 0.5));
    static const char* const combine[] = {"hard_union", "de_combinate", "smooth_max", "smooth_inv_max",
                                          "smooth_min_lin", "smooth_min_nlin", "smooth_mix"};
    if (!tag(in->get("combine_mode"), combine, 7, 0, "combine_mode", &out->combine_mode)) return false;
    out->hidden = boolean(in->get("visible"), true) ? 0 : 1;
    out->hybrid_base_iters = int32_t(num(in->get("hybrid_base_iters"), 0.0));
    out->hybrid_total_iters = int32_t(num(in->get("hybrid_total_iters"), 0.0));
    const JVal* mixins = in->get("mixins");
    if (mixins && mixins->kind == JVal::ARR) {
      out->mixin_count = int32_t(std::min<size_t>(mixins->arr.size(), ND_MAX_MIXINS));
      for (int j = 0; j < out->mixin_count; ++j) {
        const JVal& m = mixins->arr[j];
        char mw[48];
        snprintf(mw, sizeof(mw), "%s.mixins[%d]", what, j);
        if (!formula(m.get("formula"), mw, &out->mixins[j].formula, out->mixins[j].params)) return false;
        out->mixins[j].iterations = int32_t(num(m.get("iterations"), 1.0));
      }
    }
    return trap(in->get("trap"), &out->trap);
  }

  bool load(const JVal& root, int32_t width, int32_t height, nd_view_desc* view, nd_scene_desc* scene,
            int32_t* needs_scene) {
    if (root.kind != JVal::OBJ) return fail("a scene file is a JSON object");
    if (num(root.get("version"), 12) > 12) return fail("Scene file is from a newer version of the app.");
    const JVal* cam = root.get("camera");
    double pos[3], fwd[3], up[3];
    if (!cam || !vec3(cam->get("position"), "camera.position", pos) ||
        !vec3(cam->get("forward"), "camera.forward", fwd) || !vec3(cam->get("up"), "camera.up", up))
      return err.empty() ? fail("missing camera") : false;
    if (width <= 0 || height <= 0) {
      width = int32_t(num(root.get("export_width"), 0));
      height = int32_t(num(root.get("export_height"), 0));
    }
    if (width <= 0 || height <= 0) return fail("no frame size: pass one or save export_width / export_height");
    const JVal* ins = root.get("instances");
    if (!ins || ins->kind != JVal::ARR || ins->arr.empty()) return fail("the scene has no instances");
    memset(scene, 0, sizeof(*scene));
    scene->instance_count = int32_t(std::min<size_t>(ins->arr.size(), ND_MAX_INSTANCES));
    for (int i = 0; i < scene->instance_count; ++i)
      if (!instance(&ins->arr[i], i, &scene->instances[i])) return false;
    // the bench export's march settings: render_settings (RenderSettingsState and its
    // MarchPrecision, render_precision.zig:3-35), high quality on
    const JVal* rs = root.get("render_settings");
    const JVal* none = nullptr;
    auto rg = [&](const char* k) { return rs && rs->kind == JVal::OBJ ? rs->get(k) : none; };
    const JVal* pr = rg("precision");
    auto pg = [&](const char* k) { return pr && pr->kind == JVal::OBJ ? pr->get(k) : none; };
    memset(view, 0, sizeof(*view));
    // the camera is f32 in the reference (Vec3)
    float f[3], u[3];
    for (int a = 0; a < 3; ++a) {
      view->cam_pos[a] = double(float(pos[a]));
      f[a] = float(fwd[a]);
      u[a] = float(up[a]);
      view->fwd[a] = f[a];
      view->up[a] = u[a];
    }
    // FreeCamera.basis (camera.zig:103-106): right = normalize(forward x up); the
    // shaders use forward, right and up unscaled (a 90 degree vertical field of view)
    const float r[3] = {f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]};
    const float rl = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    for (int a = 0; a < 3; ++a) view->right[a] = rl < 1e-6f ? 0.0 : double(r[a] * (1.0f / rl));
    view->width = view->tile_w = width;
    view->height = view->tile_h = height;
    view->spp = 1;
    const nd_instance_desc& first = scene->instances[0];
    view->formula = first.formula;
    memcpy(view->params, first.params, sizeof(view->params));
    view->trap = first.trap;
    view->step_safety = first.step_safety;
    view->max_steps = int32_t(num(rg("max_steps"), 256));
    view->max_dist = float(num(rg("max_dist"), 24.0));
    view->eps_coef = float(num(pg("epsilon_coefficient"), 0.0005));
    view->eps_floor = float(num(pg("epsilon_floor"), 0.00005));
    view->hq_footprint_px = float(num(pg("hq_footprint_budget_px"), 2.0));
    view->refine_budget = int32_t(num(pg("refine_hq"), 20));
    view->march_verify = boolean(pg("verify_each_step"), false) ? 1 : 0;
    view->high_quality = 1;
    view->normal_mode = ND_NORMAL_TETRA;
    view->shadow_k = 16.0f;
    view->accel_levels = 6;
    view->accel_safety = 0.92f;
    // one visible instance at the identity placement without mixins is the view's
    // own formula; anything else needs the scene
    bool identity = scene->instance_count == 1 && first.mixin_count == 0 && !first.hidden;
    for (int a = 0; a < 3; ++a) identity &= first.offset[a] == 0.0f && first.scale[a] == 1.0f;
    const float eye[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int k = 0; k < 9; ++k) identity &= fabsf(first.frame[k] - eye[k]) == 0.0f;
    *needs_scene = identity ? 0 : 1;
    return true;
  }
};

// The lite-shading descriptor of a scene file: one instance's colour stops
// (ColorStopState: position, color, glossiness, ior) and the visible point and global
// lights (LightState.toGpu, scene_state.zig:594-612: a global light's direction, a
// point light's position; ray lights are not part of the lite pass and are left out).
bool load_lite(const JVal& root, int instance, nd_lite_desc* out, std::string* err) {
  memset(out, 0, sizeof(*out));
  out->ambient_occlusion = 1;
  out->specular = 1;
  out->background[0] = 0.10f;  // SIMPLE_BACKGROUND (tpl:4419); the sky is not part of this pass
  out->background[1] = 0.11f;
  out->background[2] = 0.13f;
  const JVal* ins = root.kind == JVal::OBJ ? root.get("instances") : nullptr;
  if (!ins || ins->kind != JVal::ARR || instance < 0 || size_t(instance) >= ins->arr.size()) {
    *err = "no such instance";
    return false;
  }
  const JVal* colors = ins->arr[instance].get("colors");
  if (colors && colors->kind == JVal::ARR)
    for (const JVal& c : colors->arr) {
      if (out->color_count >= ND_MAX_COLOR_STOPS) break;
      nd_color_stop& d = out->colors[out->color_count++];
      const JVal* rgb = c.get("color");
      for (int k = 0; k < 3; ++k)
        d.color[k] = rgb && rgb->kind == JVal::ARR && rgb->arr.size() > size_t(k) ? float(Loader::num(&rgb->arr[k], 0.5)) : 0.5f;
      d.position = float(Loader::num(c.get("position"), 0.0));
      d.glossiness = float(Loader::num(c.get("glossiness"), 0.0));
      d.ior = float(Loader::num(c.get("ior"), 1.5));
    }
  const JVal* lights = root.get("lights");
  if (lights && lights->kind == JVal::ARR)
    for (const JVal& l : lights->arr) {
      if (out->light_count >= ND_MAX_LIGHTS) break;
      if (!Loader::boolean(l.get("visible"), true)) continue;
      const JVal* kind = l.get("kind");
      const std::string k = kind && kind->kind == JVal::STR ? kind->str : "global";
      if (k != "point" && k != "global") continue;
      nd_light& d = out->lights[out->light_count++];
      d.type = k == "point" ? ND_LIGHT_POINT : ND_LIGHT_GLOBAL;
      const JVal* rgb = l.get("color");
      for (int q = 0; q < 3; ++q)
        d.color[q] = rgb && rgb->kind == JVal::ARR && rgb->arr.size() > size_t(q) ? float(Loader::num(&rgb->arr[q], 1.0)) : 1.0f;
      d.brightness = float(Loader::num(l.get("brightness"), 1.0));
      const double zero[3] = {0, 0, 0};
      Loader::vec3_or(l.get(d.type == ND_LIGHT_POINT ? "position" : "direction"), zero, d.position_or_direction);
    }
  return true;
}

}  // namespace

extern "C" nd_status nd_scene_file_lite(const char* json, size_t len, int32_t instance, nd_lite_desc* lite, char* err,
                                        size_t err_len) {
  std::string msg;
  JVal root;
  JsonParser p(json ? json : "", json ? len : 0);
  nd_status st = ND_OK;
  if (!json || !lite) {
    msg = "bad arguments";
    st = ND_ERR_INVALID;
  } else if (!p.parse(&root)) {
    msg = p.error();
    st = ND_ERR_INVALID;
  } else if (!load_lite(root, instance, lite, &msg)) {
    st = ND_ERR_INVALID;
  }
  if (err && err_len) {
    const size_t n = std::min(err_len - 1, msg.size());
    memcpy(err, msg.data(), n);
    err[n] = 0;
  }
  return st;
}

extern "C" nd_status nd_scene_file_load(const char* json, size_t len, int32_t width, int32_t height,
                                        nd_view_desc* view, nd_scene_desc* scene, int32_t* needs_scene, char* err,
                                        size_t err_len) {
  auto report = [&](const std::string& m) {
    if (err && err_len) {
      const size_t n = std::min(err_len - 1, m.size());
      memcpy(err, m.data(), n);
      err[n] = 0;
    }
  };
  if (!json || !view || !scene || !needs_scene) {
    report("bad arguments");
    return ND_ERR_INVALID;
  }
  JVal root;
  JsonParser p(json, len);
  if (!p.parse(&root)) {
    report(p.error());
    return ND_ERR_INVALID;
  }
  Loader L;
  if (!L.load(root, width, height, view, scene, needs_scene)) {
    report(L.err);
    return L.err.find("not in this build") != std::string::npos ? ND_ERR_NOT_FOUND
           : L.err.find("newer version") != std::string::npos ? ND_ERR_UNSUPPORTED
                                                              : ND_ERR_INVALID;
  }
  report("");
  return ND_OK;
}
