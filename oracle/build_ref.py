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
    helpers = translate_module(helper_module(template, list(TEMPLATE_FUNCS)), "ndref_tpl", contract=False)
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
    lines = ['// reference formula code, mechanically translated (generated; do not edit)',
             '#include <stdint.h>', '#include <string.h>', '#include "nd_wgsl.h"', helpers] + units
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
    src = os.path.join(OUT, "ref_formulas.cpp")
    with open(src, "w", encoding="utf-8") as fh:
        fh.write("\n".join(lines))
    cmd = ["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-ffp-contract=off",
           "-I", os.path.join(ROOT, "numericdream_b200", "csrc"), src, "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
