"""Build of the CUDA library numericdream_b200/libnd_march.so.

Steps (each incremental on file contents/mtimes):
  1. collect formula plugins (WGSL) from the formula directories;
  2. translate each with the WGSL-subset translator into a C++ namespace;
  3. emit one CUDA translation unit per formula (its kernel instantiations), one
     per formula group (mixed-formula batches in one launch) and the registry;
  4. nvcc every unit for sm_100a in parallel and link the shared library.

Formula directories: ``ND_FORMULA_DIRS`` (os.pathsep-separated list of
directories or single .wgsl files).  When unset, the build uses NumericDream's
own formula collection and built-in Mandelbulb if a NumericDream checkout is
found at ``ND_REFERENCE`` (default: the read-only checkout this build was set up
against), plus this package's ``formulas/`` directory.  ``ND_FORMULAS`` limits the
build to a comma-separated list of formula names.
"""

from __future__ import annotations

import concurrent.futures as cf
import hashlib
import json
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
GEN = os.path.join(PKG, "_generated")
OBJ = os.path.join(GEN, "obj")
LIB = os.path.join(PKG, "libnd_march.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The FP32 DE is compiled with the GPU's fast division, square root and
# transcendental approximations (--use_fast_math), which are within WGSL's own f32
# accuracy requirements (e.g. 2.5 ulp division, 2^-11 absolute sin/cos on
# [-pi, pi]), and with the polynomial acos / atan2 of nd_wgsl.h; ND_ACCURATE_MATH=1
# builds CUDA's correctly rounded / few-ulp versions instead.  FP64 DEs and the FP64 march bookkeeping are unaffected, and
# eps(t) uses explicitly rounded operations either way.
MATHFLAGS = ["-DND_ACCURATE_MATH"] if os.environ.get("ND_ACCURATE_MATH") == "1" else ["--use_fast_math"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "--expt-relaxed-constexpr",
           "-I", CSRC, "-I", INCLUDE, "-I", GEN] + MATHFLAGS + os.environ.get("ND_NVCC_EXTRA", "").split()

# Mixed-formula batches run in ONE persistent launch when every formula of the
# batch belongs to a compiled group.  The default group holds the four formulas
# of the batched benchmark (Mandelbulb, Mandelbox, Menger sponge, pseudo-Kleinian).
DEFAULT_GROUPS = {"mixed4": ["mandelbrot", "amazingbox_box", "menger3_ifs", "pseudokleinian_kleinian"],
                  # scenes of fractals standing on / beside primitives, as the
                  # reference's bench scenes are built (a call takes the first group
                  # that covers it, so the benchmark batches still use mixed4)
                  "scenes6": ["mandelbrot", "amazingbox_box", "menger3_ifs", "pseudokleinian_kleinian",
                              "sphere_primitive", "cube_primitive"]}
# Groups also carry the multi-instance scene kernels: a scene's formulas (instances
# and mixins) must all lie in one group.  ND_GROUPS adds groups:
# "name=f1,f2,...;name2=..." (formula file stems).
for _spec in filter(None, os.environ.get("ND_GROUPS", "").split(";")):
    _name, _, _members = _spec.partition("=")
    DEFAULT_GROUPS[_name.strip()] = [m.strip() for m in _members.split(",") if m.strip()]


def reference_root():
    env = os.environ.get("ND_REFERENCE")
    if env:
        return env if os.path.isdir(env) else None
    guess = os.path.join(os.sep, "root", "reference")
    return guess if os.path.isdir(os.path.join(guess, "formulas")) else None


def formula_sources() -> dict:
    """name -> (path, source text).  Later directories override earlier ones."""
    entries = []
    env = os.environ.get("ND_FORMULA_DIRS")
    if env:
        entries = [e for e in env.split(os.pathsep) if e]
    else:
        ref = reference_root()
        if ref:
            entries.append(os.path.join(ref, "src", "gpu", "shaders", "mandelbrot.wgsl"))
            entries.append(os.path.join(ref, "formulas"))
        entries.append(os.path.join(PKG, "formulas"))
    out = {}
    for e in entries:
        files = []
        if os.path.isdir(e):
            files = sorted(os.path.join(e, f) for f in os.listdir(e) if f.endswith(".wgsl"))
        elif os.path.isfile(e):
            files = [e]
        for f in files:
            name = os.path.splitext(os.path.basename(f))[0]
            with open(f, "r", encoding="utf-8") as fh:
                out[name] = (f, fh.read())
    only = os.environ.get("ND_FORMULAS")
    if only:
        keep = {n.strip() for n in only.split(",") if n.strip()}
        out = {k: v for k, v in out.items() if k in keep}
    return out


def _write_if_changed(path: str, text: str) -> bool:
    if os.path.exists(path):
        with open(path, "r", encoding="utf-8") as fh:
            if fh.read() == text:
                return False
    with open(path + ".tmp", "w", encoding="utf-8") as fh:
        fh.write(text)
    os.replace(path + ".tmp", path)
    return True


def _cpp_str(s: str) -> str:
    return json.dumps(s)


def _traits(tf) -> str:
    ns = tf.namespace
    return f"""struct F_{ns} {{
  template <class T, class P> static ND_DEV_INLINE int32_t iterations(const P& p) {{ return {ns}::de_iterations<T, P>(p); }}
  template <class T, class P> static ND_DEV_INLINE ndw::IterCarry<T> step(ndw::IterCarry<T> c, ndw::v3<T> pos, const P& p) {{ return {ns}::de_step<T, P>(c, pos, p); }}
  template <class T, class P> static ND_DEV_INLINE T finalize(ndw::IterCarry<T> c) {{ return {ns}::de_finalize<T, P>(c); }}
}};
"""


def generate(verbose=False):
    from .translator import translate, TranslateError

    os.makedirs(GEN, exist_ok=True)
    os.makedirs(os.path.join(GEN, "formulas"), exist_ok=True)
    sources = formula_sources()
    formulas, rejected = [], {}
    for name in sorted(sources):
        path, src = sources[name]
        try:
            tf = translate(src, name)
        except TranslateError as e:
            rejected[name] = str(e)
            continue
        formulas.append(tf)
        _write_if_changed(os.path.join(GEN, "formulas", name + ".inc"),
                          f"// translated from {os.path.basename(path)} by numericdream_b200.translator\n"
                          f"#pragma once\n{tf.cpp}\n")
    index = {tf.name: i for i, tf in enumerate(formulas)}
    units = []
    for tf in formulas:
        unit = os.path.join(GEN, f"k_{tf.name}.cu")
        _write_if_changed(unit, f"""// kernels of formula {tf.name} (generated)
#include "nd_kernels.cuh"
#include "formulas/{tf.name}.inc"
{_traits(tf)}
nd::KernelTable nd_kernels_{tf.namespace}() {{ return nd::make_kernel_table<nd::FormulaSet<F_{tf.namespace}>>(); }}
int32_t nd_iterations_{tf.namespace}(const float* p) {{
  return F_{tf.namespace}::iterations<float, nd::ParamRef<float>>(nd::ParamRef<float>{{p}});
}}
""")
        units.append(unit)
    groups = []
    for gname, members in DEFAULT_GROUPS.items():
        if not all(m in index for m in members):
            continue
        incs = "\n".join(f'#include "formulas/{m}.inc"' for m in members)
        traits = "\n".join(_traits(formulas[index[m]]) for m in members)
        setargs = ", ".join(f"F_{formulas[index[m]].namespace}" for m in members)
        unit = os.path.join(GEN, f"g_{gname}.cu")
        _write_if_changed(unit, f"""// kernels of formula group {gname} (generated)
#include "nd_kernels.cuh"
{incs}
{traits}
nd::KernelTable nd_group_{gname}() {{ return nd::make_kernel_table<nd::FormulaSet<{setargs}>, true>(); }}
""")
        units.append(unit)
        groups.append((gname, [index[m] for m in members]))
    # host op-counting units (same formula code, T = counting float)
    op_units = []
    for tf in formulas:
        unit = os.path.join(GEN, f"op_{tf.name}.cpp")
        _write_if_changed(unit, f"""// op counting of formula {tf.name} (generated)
#include "nd_opcount.h"
#include "nd_rayprog.h"
#include "formulas/{tf.name}.inc"
{_traits(tf)}
extern "C" void ndop_{tf.namespace}(const nd::DevView* v, int64_t ray, ndw::OpCounts* out, uint32_t* evals) {{
  nd::count_ray<nd::FormulaSet<F_{tf.namespace}>>(*v, ray, out, evals);
}}
""")
        op_units.append(unit)
    tab = ['// op-counting table (generated)', '#include "nd_opcount.h"', '#include "nd_rayprog.h"']
    for tf in formulas:
        tab.append(f'extern "C" void ndop_{tf.namespace}(const nd::DevView*, int64_t, ndw::OpCounts*, uint32_t*);')
    tab.append("typedef void (*NdOpFn)(const nd::DevView*, int64_t, ndw::OpCounts*, uint32_t*);")
    tab.append("extern const NdOpFn nd_opcount_fns[] = {" + ", ".join(f"&ndop_{tf.namespace}" for tf in formulas) + "};")
    tab.append(f"extern const int nd_opcount_fn_count = {len(formulas)};")
    optab = os.path.join(GEN, "op_table.cpp")
    _write_if_changed(optab, "\n".join(tab) + "\n")
    op_units.append(optab)
    # registry
    lines = ['// formula registry (generated)', '#include "nd_registry.h"', "", "namespace {"]
    for tf in formulas:
        lines.append(f"}}  // namespace\nnd::KernelTable nd_kernels_{tf.namespace}();\n"
                     f"int32_t nd_iterations_{tf.namespace}(const float*);\nnamespace {{")
    for gname, _ in groups:
        lines.append(f"}}  // namespace\nnd::KernelTable nd_group_{gname}();\nnamespace {{")
    lines.append("}  // namespace")
    lines.append("const nd::FormulaEntry nd_formula_entries[] = {")
    for tf in formulas:
        ps = []
        for p in tf.params:
            ps.append(f"{{{_cpp_str(p.name)}, {p.min!r}f, {p.max!r}f, {p.default!r}f, {1 if p.integral else 0}}}")
        plist = ", ".join(ps) if ps else ""
        lines.append(f"  {{{_cpp_str(tf.name)}, 0x{tf.source_hash:016x}ull, {len(tf.params)}, {{{plist}}}, "
                     f"&nd_kernels_{tf.namespace}, &nd_iterations_{tf.namespace}}},")
    if not formulas:
        lines.append('  {"", 0ull, 0, {}, nullptr, nullptr},')
    lines.append("};")
    lines.append(f"const int nd_formula_entry_count = {len(formulas)};")
    lines.append("const nd::GroupEntry nd_group_entries[] = {")
    for gname, members in groups:
        mem = ", ".join(str(m) for m in members)
        lines.append(f"  {{{_cpp_str(gname)}, {len(members)}, {{{mem}}}, &nd_group_{gname}}},")
    if not groups:
        lines.append('  {"", 0, {}, nullptr},')
    lines.append("};")
    lines.append(f"const int nd_group_entry_count = {len(groups)};")
    reg = os.path.join(GEN, "nd_registry_table.cu")
    _write_if_changed(reg, "\n".join(lines) + "\n")
    manifest = {"formulas": [tf.name for tf in formulas], "rejected": rejected,
                "groups": {g: [formulas[i].name for i in m] for g, m in groups}}
    _write_if_changed(os.path.join(GEN, "manifest.json"), json.dumps(manifest, indent=1, sort_keys=True))
    manifest["_op_units"] = op_units
    return units, reg, manifest


def _deps_hash(paths) -> str:
    h = hashlib.sha256()
    for p in paths:
        with open(p, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def _compile(src: str, obj: str, headers: list, verbose: bool):
    stamp = obj + ".hash"
    key = _deps_hash([src] + headers) + " ".join(NVFLAGS + ARCH)
    if os.path.exists(obj) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read() == key:
                return src, None, True
    cmd = [NVCC] + ARCH + NVFLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return src, r.stdout + r.stderr, False
    with open(stamp, "w") as fh:
        fh.write(key)
    with open(obj + ".ptxas.txt", "w") as fh:
        fh.write(r.stderr)
    return src, None, False


def build(verbose: bool = False, jobs: int | None = None) -> str:
    units, reg, manifest = generate(verbose)
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "nd_march.h"))
    fheaders = {}
    for u in units:
        base = os.path.basename(u)
        incs = [os.path.join(GEN, "formulas", n + ".inc") for n in manifest["formulas"]
                if f"formulas/{n}.inc" in open(u).read()]
        fheaders[u] = headers + incs
    runtime = os.path.join(CSRC, "nd_runtime.cu")
    scene_file = os.path.join(CSRC, "nd_scene_file.cu")
    image = os.path.join(CSRC, "nd_image.cu")
    all_units = units + [reg, runtime, scene_file, image]
    fheaders[reg] = headers
    fheaders[runtime] = headers
    fheaders[scene_file] = headers
    fheaders[image] = headers
    jobs = jobs or max(1, os.cpu_count() or 1)
    objs = []
    errors = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = []
        for u in all_units:
            obj = os.path.join(OBJ, os.path.splitext(os.path.basename(u))[0] + ".o")
            objs.append(obj)
            futs.append(ex.submit(_compile, u, obj, fheaders.get(u, headers), verbose))
        for f in cf.as_completed(futs):
            src, err, cached = f.result()
            if err:
                errors.append(f"{src}:\n{err}")
            elif verbose:
                print(("cached " if cached else "built  ") + os.path.basename(src), flush=True)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    link_key = _deps_hash(objs)
    stamp = LIB + ".hash"
    if not (os.path.exists(LIB) and os.path.exists(stamp) and open(stamp).read() == link_key):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
        with open(stamp, "w") as fh:
            fh.write(link_key)
    build_opcount(manifest["_op_units"], headers, jobs)
    return LIB


OPLIB = os.path.join(PKG, "libnd_opcount.so")
# ND_OPCOUNT_BUILD: the helpers take their branchy form, so that the count is of the
# operations the reference's algorithm performs (the GPU build computes both sides of
# some tests and selects, which gives the same values with fewer warp splits)
CXXFLAGS = ["-std=c++17", "-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-DND_OPCOUNT_BUILD", "-I", CSRC,
            "-I", INCLUDE, "-I", GEN]


def _compile_host(src, obj, headers):
    stamp = obj + ".hash"
    key = _deps_hash([src] + headers) + " ".join(CXXFLAGS)
    if os.path.exists(obj) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read() == key:
                return src, None
    r = subprocess.run(["g++"] + CXXFLAGS + ["-c", src, "-o", obj], capture_output=True, text=True)
    if r.returncode != 0:
        return src, r.stdout + r.stderr
    with open(stamp, "w") as fh:
        fh.write(key)
    return src, None


def build_opcount(op_units, headers, jobs):
    """Host library that counts the algorithmic FP32 ops of the ray program."""
    api = os.path.join(CSRC, "nd_opcount.cpp")
    srcs = op_units + [api]
    objs, errors = [], []
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = []
        for u in srcs:
            obj = os.path.join(OBJ, "host_" + os.path.splitext(os.path.basename(u))[0] + ".o")
            objs.append(obj)
            incs = list(headers)
            if os.path.basename(u).startswith("op_") and u != api:
                name = os.path.basename(u)[3:-4]
                inc = os.path.join(GEN, "formulas", name + ".inc")
                if os.path.exists(inc):
                    incs.append(inc)
            futs.append(ex.submit(_compile_host, u, obj, incs))
        for f in cf.as_completed(futs):
            src, err = f.result()
            if err:
                errors.append(f"{src}:\n{err}")
    if errors:
        raise RuntimeError("g++ failed:\n" + "\n".join(errors))
    key = _deps_hash(objs)
    stamp = OPLIB + ".hash"
    if not (os.path.exists(OPLIB) and os.path.exists(stamp) and open(stamp).read() == key):
        subprocess.run(["g++", "-shared", "-fopenmp", "-o", OPLIB + ".tmp"] + objs, check=True)
        os.replace(OPLIB + ".tmp", OPLIB)
        with open(stamp, "w") as fh:
            fh.write(key)
    return OPLIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
