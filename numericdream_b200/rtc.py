"""Run-time compilation of one formula plugin (the compile worker behind
nd_formula_register).

The reference compiles an edited formula on a worker thread: it splices the source
into its shader template and hands the module to the driver
(FractalRenderer.rebuildAsync, src/gpu/fractal_renderer.zig:2951, compileWorker
:1609).  Here the same source goes through the build's WGSL translator and nvcc into
a small shared library holding that formula's forward kernels (march, surface and
shadow passes, DE at points; FP32 and FP64), which the library then loads.

    python -m numericdream_b200.rtc SOURCE.wgsl OUT_DIR

Writes OUT_DIR/formula.so, whose nd_rtc_entry() returns the formula's registry entry
(name ``user_<source hash>``, @param table, kernel table, host de_iterations).  Exit
status: 0 built; 2 the translator refused the source; 3 nvcc failed.  The message of
a failure is in OUT_DIR/error.txt.
"""

from __future__ import annotations

import os
import subprocess
import sys

from . import build
from .formula import source_hash
from .translator import TranslateError, translate


def unit_source(tf) -> str:
    params = ", ".join(f"{{{build._cpp_str(p.name)}, {p.min!r}f, {p.max!r}f, {p.default!r}f, {1 if p.integral else 0}}}"
                       for p in tf.params)
    ns = tf.namespace
    return f"""// formula {tf.name}, compiled at run time by numericdream_b200.rtc (generated)
#include "nd_registry.h"
#include "formulas/{tf.name}.inc"
{build._traits(tf)}
namespace {{
nd::KernelTable kernels() {{ return nd::make_kernel_table<nd::FormulaSet<F_{ns}>, false, true>(); }}
int32_t iterations(const float* p) {{ return F_{ns}::iterations<float, nd::ParamRef<float>>(nd::ParamRef<float>{{p}}); }}
const nd::FormulaEntry entry = {{{build._cpp_str(tf.name)}, 0x{tf.source_hash:016x}ull, {len(tf.params)}, {{{params}}},
                                 &kernels, &iterations}};
}}  // namespace
extern "C" const nd::FormulaEntry* nd_rtc_entry() {{ return &entry; }}
"""


def compile_formula(src: str, out_dir: str) -> int:
    name = f"user_{source_hash(src):016x}"
    os.makedirs(os.path.join(out_dir, "formulas"), exist_ok=True)
    err = os.path.join(out_dir, "error.txt")
    try:
        tf = translate(src, name)
    except TranslateError as e:
        with open(err, "w") as fh:
            fh.write(str(e))
        return 2
    with open(os.path.join(out_dir, "formulas", name + ".inc"), "w") as fh:
        fh.write(f"#pragma once\n{tf.cpp}\n")
    unit = os.path.join(out_dir, "formula.cu")
    with open(unit, "w") as fh:
        fh.write(unit_source(tf))
    lib = os.path.join(out_dir, "formula.so")
    cmd = ([build.NVCC] + build.ARCH +
           ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", build.CSRC,
            "-I", build.INCLUDE, "-I", out_dir] + build.MATHFLAGS + ["-shared", "-o", lib, unit, "-lcudart"])
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        with open(err, "w") as fh:
            fh.write("nvcc failed:\n" + r.stdout + r.stderr)
        return 3
    return 0


def main(argv) -> int:
    if len(argv) != 3:
        print(__doc__, file=sys.stderr)
        return 64
    with open(argv[1], "r", encoding="utf-8", newline="") as fh:  # the exact bytes: their hash is the key
        src = fh.read()
    return compile_formula(src, argv[2])


if __name__ == "__main__":
    sys.exit(main(sys.argv))
