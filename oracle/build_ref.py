"""Recipe for oracle/_ref: the reference's own formula code, compiled for the host.

TEST INFRASTRUCTURE.  NumericDream's DE code is WGSL, which only runs through a
graphics API (unavailable on this box).  This recipe reads the reference's WGSL where
it lies -- every formula file, the built-in Mandelbulb and the DE helper functions of
the shader template (box_fold, sphere_fold, bulb_power_step, rotate_xyz_deg, ...) --
translates it mechanically with the build's WGSL translator (helpers included, so no
hand-written code stands between the reference text and the compiled program except
the WGSL builtins), and compiles oracle/_ref/libref_formulas.so with g++.  Nothing
from the reference is copied into the repository: outputs go to oracle/_ref/ only
(git-ignored).

The library gives DE values of each reference formula at given points in FP64 or
FP32.  tests/golden/make_golden.py uses it to write the committed fixtures that pin
the hand-written oracle and the CUDA path; it only runs where the reference exists.
"""

from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libref_formulas.so")


def reference_root():
    env = os.environ.get("ND_REFERENCE")
    if env:
        return env if os.path.isdir(env) else None
    guess = os.path.join(os.sep, "root", "reference")
    return guess if os.path.isdir(os.path.join(guess, "formulas")) else None


def _extract_fn(text: str, name: str) -> str:
    m = re.search(r"^fn\s+" + re.escape(name) + r"\s*\(", text, re.M)
    if not m:
        raise KeyError(name)
    i = text.index("{", m.end())
    depth = 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[m.start():j + 1]
    raise ValueError(name)


def helper_module(template: str, names) -> str:
    """The helper functions named, plus every single-line module-level const the
    translator accepts (only the ones the helpers use are ever evaluated)."""
    sys.path.insert(0, ROOT)
    from numericdream_b200.translator.wgsl import Parser, lex, TranslateError

    parts = []
    for line in template.split("\n"):
        if line.startswith("const ") and line.rstrip().endswith(";") and "u." not in line:
            try:
                Parser(lex(line)).module()
            except TranslateError:
                continue
            parts.append(line)
    for n in names:
        parts.append(_extract_fn(template, n))
    return "\n".join(parts) + "\n"


# The march of the path, from the shader template: march_epsilon (tpl:1813-1815),
# march_to (tpl:1859-1963) and tetra_gradient (tpl:1790-1804).  The text is rewritten
# only where the template reaches state outside the function, so that the functions
# translate on their own: uniform fields become entries of a settings array m
# (MARCH_SETTINGS), the coarse-march and overstep-watch switches (module-scope
# private variables, false for this pass) become false, warp_step_limit and
# accel_skip (warps off, accelerator off) become their off values, scene_de(pos)
# gains the parameter arrays, and MarchResult(hit, dist, steps, evals) is returned
# as a vec4f.
MARCH_FUNCS = ["march_epsilon", "march_to", "tetra_gradient"]
MARCH_SETTINGS = {"u.resolution.y": 8, "u.epsilon_coefficient": 0, "u.epsilon_floor": 1, "u.max_steps": 2,
                  "u.refine_fast": 3, "u.refine_hq": 4, "u.high_quality": 5, "u.march_verify": 6,
                  "u.hq_footprint_budget_px": 7}
# m[9]: the instance DE factor clamp(step_safety, 0.001, 1) (instance_de_factor
# tpl:1617-1620 with scale 1)
MARCH_FORMULAS = ["mandelbrot", "amazingbox_box", "menger3_ifs", "pseudokleinian_kleinian", "sphere_primitive",
                  "cube_primitive"]
MARCH_PRELUDE = """
fn march_result(h: bool, d: f32, s: f32, e: f32) -> vec4f { return vec4f(select(0.0, 1.0, h), d, s, e); }
fn scene_de(pos: vec3f, p: Params, m: Params) -> f32 {
    var c = IterCarry(pos, 1.0);
    let n = de_iterations(p);
    for (var i = 0; i < n; i++) { c = de_step(c, pos, p); }
    return de_finalize(c) * m[9];
}
"""


def march_module(template: str) -> str:
    """march_epsilon, march_to and tetra_gradient of the template, rewritten as above."""
    sigs = {"march_epsilon": ("(t: f32)", "(t: f32, m: Params)"),
            "march_to": ("(origin: vec3f, dir: vec3f, max_t: f32)",
                         "(origin: vec3f, dir: vec3f, max_t: f32, p: Params, m: Params)"),
            "tetra_gradient": ("(pos: vec3f, e: f32)", "(pos: vec3f, e: f32, p: Params, m: Params)")}
    out = []
    for name in MARCH_FUNCS:
        fn = _extract_fn(template, name)
        old, new = sigs[name]
        if old not in fn:
            raise ValueError(f"{name}: unexpected signature")
        fn = fn.replace(old, new)
        for field, k in MARCH_SETTINGS.items():
            fn = fn.replace(field, f"m[{k}]")
        fn = fn.replace("g_coarse_march", "false").replace("g_overstep_watch", "false")
        fn = re.sub(r"^\s*g_overstep_(worst|count)\s*\+?=.*;\s*$", "", fn, flags=re.M)
        fn = re.sub(r"warp_step_limit\([^()]*\)", "INFINITE_DISTANCE", fn)
        fn = re.sub(r"accel_skip\([^()]*\)", "0.0", fn)
        fn = re.sub(r"(?<!fn )\bscene_de\(([^()]*(?:\([^()]*\)[^()]*)*)\)", r"scene_de(\1, p, m)", fn)
        fn = re.sub(r"(?<!fn )\bmarch_epsilon\(([^()]*)\)", r"march_epsilon(\1, m)", fn)
        fn = fn.replace("-> MarchResult", "-> vec4f").replace("MarchResult(", "march_result(")
        if re.search(r"\bu\.[a-z]", fn):
            raise ValueError(f"{name}: a uniform field is not mapped")
        out.append(fn)
    consts = [l for l in template.split("\n")
              if re.match(r"^const (INFINITE_DISTANCE|COARSE_[A-Z_]+|OVERSTEP_TOLERANCE|TETRAHEDRAL_TAPS)\b", l)]
    return "\n".join(consts) + "\n" + MARCH_PRELUDE + "\n".join(out) + "\n"


# The orbit trap of the formula wrapper: orbit_trap_distance / _begin / _update /
# _finish (tpl:1227-1289) with the OrbitTrap record passed as an array t (center xyz,
# shape, box xyz, mode, radius, tube: TRAP_FIELDS), and the per-formula wrapper that
# the reference generates (appendFormulaWrapper, fractal_renderer.zig:490-512), read
# from the Zig source, with the distance LOD off (lod_iterations(n) = (n, 1), so
# lod_blend gives the full-iteration carry) and the trap record as a parameter.
TRAP_FUNCS = ["orbit_trap_distance", "orbit_trap_begin", "orbit_trap_update", "orbit_trap_finish"]
TRAP_FIELDS = {"t.center": "vec3f(t[0], t[1], t[2])", "t.shape": "i32(t[3])", "t.box": "vec3f(t[4], t[5], t[6])",
               "t.mode": "i32(t[7])", "t.radius": "t[8]", "t.tube": "t[9]"}


def trap_module(template: str, renderer_zig: str) -> str:
    out = [l for l in template.split("\n") if re.match(r"^const TRAP_[A-Z_]+ = ", l)]
    for name in TRAP_FUNCS:
        fn = _extract_fn(template, name).replace("t: OrbitTrap", "t: Params")
        for field, expr in TRAP_FIELDS.items():
            fn = fn.replace(field, expr)
        out.append(fn)
    m = re.search(r"fn appendFormulaWrapper\(.*?\n(.*?)\n\s*, \.\{code\}\);", renderer_zig, re.S)
    if not m:
        raise ValueError("appendFormulaWrapper not found")
    body = "\n".join(l.split("\\\\", 1)[1] for l in m.group(1).split("\n") if "\\\\" in l)
    body = body.replace("{{", "{").replace("}}", "}").replace("_{0}", "")
    body = body.replace("fn formula(pos: vec3f, p: Params, slot: i32)", "fn formula_trap(pos: vec3f, p: Params, t: Params)")
    body = re.sub(r"^\s*g_image_slot = .*;\s*$", "", body, flags=re.M)
    body = re.sub(r"^\s*let trap_spec = orbit_trap\(slot\);\s*$", "", body, flags=re.M).replace("trap_spec", "t")
    body = re.sub(r"lod_iterations\(([^()]*\([^()]*\))\)", r"vec2f(f32(\1), 1.0)", body)
    body = body.replace("lod_blend(carry_lo, carry, lod.y)", "carry")
    if "slot" in body or "lod_" in body or "formula_trap" not in body:
        raise ValueError("unexpected formula wrapper text")
    out.append(body)
    return "\n".join(out) + "\n"


# The shadow ray: visibility_march (tpl:2282-2342) for an opaque scene (the
# reference's scene_has_transparency false, photons and fake caustics off: the
# transparent-hit branch is cut, and the spectral tint, which stays 1 then, becomes
# an f32), its VisParams record passed as an array (VIS_FIELDS), built by the driver
# from the template's SHADOW_* constants in shadow_factor's order (tpl:2365-2375,
# checked against the template text).  And the Lambert level of simple_geometry
# (tpl:4492-4507): its key_dir / lambert / shade statements.
VIS_FIELDS = ["k", "t0", "hit_eps", "exit_slope", "exit_bias", "step_floor", "floor_growth", "min_step", "tint_cut"]
SHADOW_ARGS = ["mix(light.shadow_softness, SHADOW_HARD_K, light.hard_shadows)", "bias", "SHADOW_HIT_EPS",
               "SHADOW_EXIT_SLOPE", "SHADOW_EXIT_BIAS", "SHADOW_STEP_FLOOR", "SHADOW_FLOOR_GROWTH", "SHADOW_MIN_STEP",
               "SHADOW_TINT_CUT", "min(i32(u.max_steps), SHADOW_MAX_STEPS)", "true"]


def shadow_module(template: str):
    """visibility_march and the simple shade as WGSL, and the SHADOW_* constants."""
    sf = _extract_fn(template, "shadow_factor")
    m = re.search(r"VisParams\((.*)\);", sf)
    args = [a.strip() for a in re.split(r",(?![^()]*\))", m.group(1))] if m else []
    if args != SHADOW_ARGS or "let bias = SHADOW_BIAS;" not in sf:
        raise ValueError("shadow_factor builds VisParams differently than expected")
    consts = {}
    for name in ("SHADOW_BIAS", "SHADOW_HIT_EPS", "SHADOW_EXIT_SLOPE", "SHADOW_EXIT_BIAS", "SHADOW_STEP_FLOOR",
                 "SHADOW_FLOOR_GROWTH", "SHADOW_MIN_STEP", "SHADOW_TINT_CUT", "SHADOW_MAX_STEPS"):
        c = re.search(r"^const " + name + r"\s*=\s*([0-9.eE+-]+);", template, re.M)
        consts[name] = c.group(1)
    fn = _extract_fn(template, "visibility_march")
    old_sig = "(origin: vec3f, light_dir: vec3f, light_dist: f32, vp: VisParams) -> Spec"
    if old_sig not in fn:
        raise ValueError("visibility_march: unexpected signature")
    fn = fn.replace(old_sig, "(origin: vec3f, light_dir: vec3f, light_dist: f32, vp: Params, fp: Params, m: Params) -> f32")
    for i, f in enumerate(VIS_FIELDS):
        fn = re.sub(r"\bvp\." + f + r"\b", f"vp[{i}]", fn)
    fn = fn.replace("vp.steps", "i32(vp[9])").replace("vp.caustics", "(vp[10] > 0.5)")
    fn = fn.replace("approx_on(APPROX_FAKE_CAUSTICS)", "false").replace("photons_on()", "false")
    fn = fn.replace("!scene_has_transparency", "true")
    fn = re.sub(r"let mat = hit_material\(p\)\.mat;.*?(?=\n\s*in_solid = true;)", "", fn, flags=re.S)
    fn = fn.replace("spec_splat(", "(").replace("spec_scale(tint, ", "tint * (")
    fn = re.sub(r"accel_skip\([^()]*\)", "0.0", fn)
    fn = re.sub(r"(?<!fn )\bscene_de\(([^()]*)\)", r"scene_de(\1, fp, m)", fn)
    if re.search(r"\bspec_\w+\(|\bhit_material\(|\bfake_caustic\(|\bu\.[a-z]|VisParams|\bSpec\b", fn):
        raise ValueError("visibility_march: unexpected reach outside the function")
    sg = _extract_fn(template, "simple_geometry")
    stmts = [re.search(r"^\s*let " + v + r" = .*;$", sg, re.M) for v in ("key_dir", "lambert", "shade")]
    if not all(stmts):
        raise ValueError("simple_geometry: unexpected text")
    body = "\n".join(x.group(0) for x in stmts).replace("u.camera_up", "cam_up").replace("u.camera_right", "cam_right")
    shade = ("fn simple_shade(dir: vec3f, normal: vec3f, cam_up: vec3f, cam_right: vec3f) -> f32 {\n" + body +
             "\n    return shade;\n}\n")
    simple_consts = [l for l in template.split("\n") if re.match(r"^const SIMPLE_(AMBIENT|KEY_UP|KEY_LEFT) = ", l)]
    return "\n".join(simple_consts) + "\n" + fn + "\n" + shade, consts


# Pieces of the lite shading: calc_ao (tpl:1825-1840, the ambient-occlusion part
# switched on, its hotspot bookkeeping dropped), fresnel_schlick (tpl:3424-3430) and
# orbit_trap_to_strip (tpl:2025-2035, the instance's span / offset / repeat passed as
# an array s).
def lite_module(template: str) -> str:
    ao = _extract_fn(template, "calc_ao").replace("(pos: vec3f, normal: vec3f, t: f32)",
                                                  "(pos: vec3f, normal: vec3f, t: f32, p: Params, m: Params)")
    ao = ao.replace("!part_on(PART_AMBIENT_OCCLUSION)", "false")
    ao = re.sub(r"^\s*(let hot_prev = hot_enter\(.*\);|g_hot_src = hot_prev;)\s*$", "", ao, flags=re.M)
    ao = re.sub(r"(?<!fn )\bscene_de\(([^()]*)\)", r"scene_de(\1, p, m)", ao)
    st = _extract_fn(template, "orbit_trap_to_strip").replace("(slot: i32, v: f32)", "(s: Params, v: f32)")
    for field, k in (("trap_span", 0), ("trap_offset", 1), ("trap_repeat", 2)):
        st = st.replace(f"u.instances[slot].{field}", f"s[{k}]")
    fr = _extract_fn(template, "fresnel_schlick")
    for name, fn in (("calc_ao", ao), ("orbit_trap_to_strip", st)):
        if re.search(r"\bu\.|hot_|part_on|slot", fn):
            raise ValueError(f"{name}: unexpected reach outside the function")
    consts = [l for l in template.split("\n") if re.match(r"^const (AO_[A-Z_]+|TRAP_MIN_SPAN|TRAP_STRIP_[A-Z]+) = ", l)]
    return "\n".join(consts) + "\n" + ao + "\n" + st + "\n" + fr + "\n"


MARCH_DRIVER = """
template <class T> struct RefMarchParams {
  const float* v;
  T operator[](int i) const { return T(v[i]); }
};
// One primary ray of the fs_simple pass (tpl:4522-4538): pixel centre, tile
// transform, dir = normalize(forward + uv.x right + uv.y up), march_to to max_dist,
// and at a hit normalize(tetra_gradient(p, march_epsilon(t))), simple_geometry's
// Lambert level with the camera key light and, when the view has a shadow ray, the
// visibility toward its LIGHT_GLOBAL light (light_sample_ex: distance 2 max_dist)
// from p + n SHADOW_BIAS.  out[12]: hit, t, steps, evals (march), normal xyz, normal
// evals, shade, shadow visibility (1 without a shadow ray), 0, 0.
template <class T, class F>
static void ref_trace_ray(const nd_view_desc& v, const float* prm, const float* m, const float* vis, int64_t local,
                          F&& fns, double* out) {
  using V = ndw::v3<T>;
  const int64_t npix = int64_t(v.tile_w) * v.tile_h;
  const int64_t pix = local % npix;
  const T px = T(v.tile_x + int(pix % v.tile_w)) + T(0.5), py = T(v.tile_y + int(pix / v.tile_w)) + T(0.5);
  const T ndc_x = px / T(v.width) * T(2) - T(1), ndc_y = T(1) - py / T(v.height) * T(2);
  const T aspect = T(v.width) / T(v.height);
  const T ux = ndc_x * aspect, uy = -ndc_y;
  const V fwd(T(v.fwd[0]), T(v.fwd[1]), T(v.fwd[2])), right(T(v.right[0]), T(v.right[1]), T(v.right[2])),
      up(T(v.up[0]), T(v.up[1]), T(v.up[2]));
  const V dir = ndw::normalize(fwd + right * ux + up * uy);
  const V org(T(v.cam_pos[0]), T(v.cam_pos[1]), T(v.cam_pos[2]));
  RefMarchParams<T> P{prm}, M{m};
  const ndw::v4<T> r = fns.march(org, dir, T(v.max_dist), P, M);
  out[0] = double(r.x); out[1] = double(r.y); out[2] = double(r.z); out[3] = double(r.w);
  for (int k = 4; k < 12; ++k) out[k] = 0.0;
  out[9] = 1.0;
  if (r.x > T(0.5)) {
    const V pos = org + dir * r.y;
    const V n = ndw::normalize(fns.gradient(pos, fns.eps(r.y, M), P, M));
    out[4] = double(n.x); out[5] = double(n.y); out[6] = double(n.z); out[7] = 4.0;
    out[8] = double(fns.shade(dir, n, up, right));
    if (v.shadow) {
      const V ld = ndw::normalize(V(T(v.light_dir[0]), T(v.light_dir[1]), T(v.light_dir[2])));
      RefMarchParams<T> VP{vis};
      const ndw::v2<T> s = fns.visibility(pos + n * T(vis[1]), ld, T(v.max_dist) * T(2), VP, P, M);
      out[9] = double(s.x);
      out[10] = double(s.y);
    }
  }
}
// VisParams of shadow_factor (tpl:2370): k = mix(softness, SHADOW_HARD_K, hard) with
// the soft light of the view (k = shadow_k), then the SHADOW_* constants.
static void ref_shadow_settings(const nd_view_desc& v, float* vis) {
  for (int i = 0; i < 16; ++i) vis[i] = 0.0f;
  vis[0] = v.shadow_k;
  vis[1] = REF_SHADOW_BIAS; vis[2] = REF_SHADOW_HIT_EPS; vis[3] = REF_SHADOW_EXIT_SLOPE;
  vis[4] = REF_SHADOW_EXIT_BIAS; vis[5] = REF_SHADOW_STEP_FLOOR; vis[6] = REF_SHADOW_FLOOR_GROWTH;
  vis[7] = REF_SHADOW_MIN_STEP; vis[8] = REF_SHADOW_TINT_CUT;
  vis[9] = float(v.max_steps < REF_SHADOW_MAX_STEPS ? v.max_steps : REF_SHADOW_MAX_STEPS);
  vis[10] = 1.0f;
}
static void ref_march_settings(const nd_view_desc& v, float* m) {
  for (int i = 0; i < 16; ++i) m[i] = 0.0f;
  m[0] = v.eps_coef; m[1] = v.eps_floor; m[2] = float(v.max_steps);
  m[3] = v.high_quality ? 0.0f : float(v.refine_budget);  // refine_fast
  m[4] = v.high_quality ? float(v.refine_budget) : 0.0f;  // refine_hq
  m[5] = float(v.high_quality); m[6] = float(v.march_verify); m[7] = v.hq_footprint_px;
  m[8] = float(v.height);
  m[9] = v.step_safety < 0.001f ? 0.001f : (v.step_safety > 1.0f ? 1.0f : v.step_safety);
}
"""


def build(force: bool = False):
    ref = reference_root()
    if ref is None:
        return None
    sys.path.insert(0, ROOT)
    from numericdream_b200.translator import translate_module, TranslateError
    from numericdream_b200.translator.wgsl import TEMPLATE_FUNCS

    tpl_path = os.path.join(ref, "src", "gpu", "shaders", "template.wgsl")
    files = {"mandelbrot": os.path.join(ref, "src", "gpu", "shaders", "mandelbrot.wgsl")}
    fdir = os.path.join(ref, "formulas")
    for f in sorted(os.listdir(fdir)):
        if f.endswith(".wgsl"):
            files[f[:-5]] = os.path.join(fdir, f)
    sources = [tpl_path] + list(files.values()) + [os.path.abspath(__file__),
                                                   os.path.join(ROOT, "numericdream_b200", "translator", "wgsl.py"),
                                                   os.path.join(ROOT, "numericdream_b200", "csrc", "nd_wgsl.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(s) for s in sources):
        return LIB
    os.makedirs(OUT, exist_ok=True)
    with open(tpl_path, encoding="utf-8") as fh:
        template = fh.read()
    helpers = translate_module(helper_module(template, list(TEMPLATE_FUNCS) + ["combine_de"]), "ndref_tpl",
                               contract=False)
    units, names = [], []
    for name, path in files.items():
        with open(path, encoding="utf-8") as fh:
            src = fh.read()
        if "@image" in src:
            continue
        ns = "ndref_" + re.sub(r"[^A-Za-z0-9_]", "_", name)
        try:
            units.append(translate_module(src, ns, helper_ns="ndref_tpl"))
        except TranslateError:
            continue
        names.append((name, ns))
    march_src = march_module(template)
    shadow_src, shadow_consts = shadow_module(template)
    march_src += "\n" + shadow_src + "\n" + lite_module(template)
    with open(os.path.join(ref, "src", "gpu", "fractal_renderer.zig"), encoding="utf-8") as fh:
        trap_src = trap_module(template, fh.read())
    march_units, march_names = [], []
    for name in MARCH_FORMULAS:
        with open(files[name], encoding="utf-8") as fh:
            src = fh.read()
        ns = "ndrefm_" + name
        march_units.append(translate_module(src + "\n" + march_src + "\n" + trap_src, ns, helper_ns="ndref_tpl"))
        march_names.append((name, ns))
    lines = ['// reference formula code, mechanically translated (generated; do not edit)',
             '#include <stdint.h>', '#include <string.h>', '#include "nd_wgsl.h"',
             '#include "../../include/nd_march.h"', helpers] + units + march_units + \
            [f"static const float REF_{k} = float({v});" for k, v in shadow_consts.items() if k != "SHADOW_MAX_STEPS"] + \
            [f"static const int REF_SHADOW_MAX_STEPS = {shadow_consts['SHADOW_MAX_STEPS']};", MARCH_DRIVER]
    lines.append("""
template <class T> struct RefParams {
  const float* v;
  T operator[](int i) const { return T(v[i]); }
};
template <class T, int K> static double ref_eval(const float* params, const double* p3);
""")
    for k, (name, ns) in enumerate(names):
        lines.append(f"""template <> double ref_eval<float, {k}>(const float* params, const double* p3) {{
  using T = float; RefParams<T> p{{params}};
  const ndw::v3<T> pos = ndw::v3<T>(T(p3[0]), T(p3[1]), T(p3[2]));
  ndw::IterCarry<T> c{{pos, T(1)}};
  int n = {ns}::de_iterations<T, RefParams<T>>(p); if (n > 4096) n = 4096;
  for (int i = 0; i < n; ++i) c = {ns}::de_step<T, RefParams<T>>(c, pos, p);
  return double({ns}::de_finalize<T, RefParams<T>>(c));
}}
template <> double ref_eval<double, {k}>(const float* params, const double* p3) {{
  using T = double; RefParams<T> p{{params}};
  const ndw::v3<T> pos = ndw::v3<T>(p3[0], p3[1], p3[2]);
  ndw::IterCarry<T> c{{pos, T(1)}};
  int n = {ns}::de_iterations<T, RefParams<T>>(p); if (n > 4096) n = 4096;
  for (int i = 0; i < n; ++i) c = {ns}::de_step<T, RefParams<T>>(c, pos, p);
  return {ns}::de_finalize<T, RefParams<T>>(c);
}}""")
    table = ",\n".join(f'  {{"{name}", &ref_eval<float, {k}>, &ref_eval<double, {k}>}}' for k, (name, _) in enumerate(names))
    lines.append(f"""
struct RefEntry {{ const char* name; double (*f32)(const float*, const double*); double (*f64)(const float*, const double*); }};
static const RefEntry kRef[] = {{
{table}
}};
extern "C" int ref_formula_count(void) {{ return {len(names)}; }}
extern "C" const char* ref_formula_name(int i) {{ return (i >= 0 && i < {len(names)}) ? kRef[i].name : nullptr; }}
// DE of a reference formula at n points (xyz triples); precision 32 or 64.
// Returns -1 for an unknown name.
extern "C" int ref_de(const char* name, const float* params, int64_t n, const double* pts, double* out, int precision) {{
  for (int k = 0; k < {len(names)}; ++k) {{
    if (strcmp(kRef[k].name, name) != 0) continue;
    for (int64_t i = 0; i < n; ++i) out[i] = precision == 32 ? kRef[k].f32(params, pts + 3 * i) : kRef[k].f64(params, pts + 3 * i);
    return 0;
  }}
  return -1;
}}
""")
    cases, trap_cases = [], []
    for k, (name, ns) in enumerate(march_names):
        lines.append(f"""struct RefMarchFns{k} {{
  template <class T, class P> ndw::v4<T> march(ndw::v3<T> o, ndw::v3<T> d, T max_t, const P& p, const P& m) const {{
    return {ns}::march_to<T, P>(o, d, max_t, p, m);
  }}
  template <class T, class P> ndw::v3<T> gradient(ndw::v3<T> pos, T e, const P& p, const P& m) const {{
    return {ns}::tetra_gradient<T, P>(pos, e, p, m);
  }}
  template <class T, class P> T eps(T t, const P& m) const {{ return {ns}::march_epsilon<T, P>(t, m); }}
  template <class T, class P> ndw::v2<T> de_trap(ndw::v3<T> pos, const P& p, const P& t) const {{
    return {ns}::formula_trap<T, P>(pos, p, t);
  }}
  template <class T> T shade(ndw::v3<T> dir, ndw::v3<T> n, ndw::v3<T> up, ndw::v3<T> right) const {{
    return {ns}::simple_shade<T, RefMarchParams<T>>(dir, n, up, right);
  }}
  template <class T, class P> T ao(ndw::v3<T> pos, ndw::v3<T> n, T t, const P& p, const P& m) const {{
    return {ns}::calc_ao<T, P>(pos, n, t, p, m);
  }}
  template <class T, class P> T strip(const P& s, T v) const {{ return {ns}::orbit_trap_to_strip<T, P>(s, v); }}
  template <class T> T fresnel(T c, T ior) const {{ return {ns}::fresnel_schlick<T, RefMarchParams<T>>(c, ior); }}
  // visibility (its DE evaluations are not counted: 0)
  template <class T, class P> ndw::v2<T> visibility(ndw::v3<T> o, ndw::v3<T> l, T dist, const P& vp, const P& p,
                                                    const P& m) const {{
    return ndw::v2<T>({ns}::visibility_march<T, P>(o, l, dist, vp, p, m), T(0));
  }}
}};""")
        trap_cases.append(f'  if (strcmp(name, "{name}") == 0) {{ RefMarchFns{k} f; for (int64_t i = 0; i < n; ++i) {{ '
                          f'if (precision == 32) {{ const auto r = f.de_trap<float>(ndw::v3<float>(float(pts[3*i]), float(pts[3*i+1]), float(pts[3*i+2])), RefMarchParams<float>{{params}}, RefMarchParams<float>{{trap}}); out2[2*i] = r.x; out2[2*i+1] = r.y; }} '
                          f'else {{ const auto r = f.de_trap<double>(ndw::v3<double>(pts[3*i], pts[3*i+1], pts[3*i+2]), RefMarchParams<double>{{params}}, RefMarchParams<double>{{trap}}); out2[2*i] = r.x; out2[2*i+1] = r.y; }} }} return 0; }}')
        cases.append(f'    if (strcmp(name, "{name}") == 0) {{ RefMarchFns{k} f; if (precision == 32) '
                     f'ref_trace_ray<float>(*v, v->params, m, vis, i, f, o); else ref_trace_ray<double>(*v, v->params, m, vis, i, f, o); continue; }}')
    ao_cases = "\n".join(f'  if (strcmp(name, "{n}") == 0) {{ RefMarchFns{k} f; for (int64_t i = 0; i < n; ++i) '
                          f'out[i] = double(f.ao<double>(ndw::v3<double>(pos[3*i], pos[3*i+1], pos[3*i+2]), '
                          f'ndw::v3<double>(nrm[3*i], nrm[3*i+1], nrm[3*i+2]), t[i], P, M)); return 0; }}'
                          for k, (n, _) in enumerate(march_names))
    lines.append("""
// calc_ao of the reference at n hit points (FP64; the view's formula and settings).
extern "C" int ref_ao(const nd_view_desc* v, const char* name, int64_t n, const double* pos, const double* nrm,
                      const double* t, double* out) {
  float m[16];
  ref_march_settings(*v, m);
  RefMarchParams<double> P{v->params}, M{m};
""" + ao_cases + """
  return -1;
}
// orbit_trap_to_strip and fresnel_schlick of the reference (f32) at n inputs.
extern "C" void ref_strip_fresnel(int64_t n, const float* span_offset_repeat, const float* v, const float* cosv,
                                  const float* ior, float* strip, float* fresnel) {
  RefMarchFns0 f;
  for (int64_t i = 0; i < n; ++i) {
    RefMarchParams<float> s{span_offset_repeat + 3 * i};
    strip[i] = f.strip<float>(s, v[i]);
    fresnel[i] = f.fresnel<float>(cosv[i], ior[i]);
  }
}
""")
    lines.append("""
// The reference's generated formula wrapper (DE and orbit trap) at n points; trap:
// center xyz, shape, box xyz, mode, radius, tube.  -1 for a formula without one.
extern "C" int ref_de_trap(const char* name, const float* params, const float* trap, int precision, int64_t n,
                           const double* pts, double* out2) {
""" + "\n".join(trap_cases) + """
  return -1;
}
""")
    lines.append("""
// The reference's fs_simple primary pass for rays [first, first + n) of a view (tile
// and spp 1 only): out[12 i ..] as ref_trace_ray.  -1 for a formula without a march.
extern "C" int ref_trace(const nd_view_desc* v, const char* name, int precision, int64_t first, int64_t n,
                         double* out) {
  float m[16], vis[16];
  ref_march_settings(*v, m);
  ref_shadow_settings(*v, vis);
  int found = 0;
""" + "\n".join(f'  found |= strcmp(name, "{n}") == 0;' for n, _ in march_names) + """
  if (!found) return -1;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t j = 0; j < n; ++j) {
    const int64_t i = first + j;
    double* o = out + 12 * j;
""" + "\n".join(cases) + """
  }
  return 0;
}
""")
    lines.append("""
// combine_de (tpl:1708-1730) of the template: (distance, material weight) of an
// instance combined into the scene so far, at n inputs (mode, d, di, k).
extern "C" void ref_combine(int64_t n, const int32_t* mode, const float* d, const float* di, const float* k,
                            float* out2) {
  for (int64_t i = 0; i < n; ++i) {
    const ndw::v2<float> r = ndref_tpl::combine_de<float, RefMarchParams<float>>(mode[i], d[i], di[i], k[i]);
    out2[2 * i] = r.x;
    out2[2 * i + 1] = r.y;
  }
}
""")
    src = os.path.join(OUT, "ref_formulas.cpp")
    with open(src, "w", encoding="utf-8") as fh:
        fh.write("\n".join(lines))
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-I", os.path.join(ROOT, "numericdream_b200", "csrc"), src, "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
