"""The C ABI from a plain C host, as NumericDream's Zig host would use it through
translate-C: include/nd_march.h compiles as strict C99 with every warning an error,
and a C program linked against the library finds a formula, reads its @param table
and its view defaults, and counts a view's rays.  None of these calls needs a GPU."""

import os
import subprocess

import pytest

from numericdream_b200 import runtime

HERE = os.path.dirname(os.path.abspath(__file__))
INCLUDE = os.path.join(HERE, "..", "include")

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "nd_march.h"

int main(void) {
  nd_formula_id id = -1;
  nd_param_info params[ND_MAX_PARAMS];
  int32_t n = 0, count = 0;
  nd_view_desc view;
  int64_t rays = 0;
  if (nd_abi_version() != ND_ABI_VERSION) return 10;
  if (nd_formula_count(&count) != ND_OK || count < 1) return 11;
  if (nd_formula_find("mandelbrot", &id) != ND_OK) return 12;
  if (nd_formula_find("no_such_formula", &id) != ND_ERR_NOT_FOUND) return 13;
  if (nd_formula_find("mandelbrot", &id) != ND_OK) return 14;
  if (nd_formula_params(id, params, &n) != ND_OK || n != 2) return 15;
  if (strcmp(params[0].name, "Power") != 0 || params[1].integral != 1) return 16;
  if (nd_view_defaults(id, &view) != ND_OK || view.formula != id) return 17;
  view.width = view.tile_w = 320;
  view.height = view.tile_h = 200;
  view.tile_x = view.tile_y = 0;
  view.spp = 4;
  if (nd_count_rays(&view, 1, &rays) != ND_OK || rays != 320 * 200 * 4) return 18;
  printf("%s %d %s %g\n", nd_status_string(ND_ERR_TIMEOUT), (int)count, params[0].name,
         (double)params[0].default_value);
  return 0;
}
"""


def test_header_compiles_as_c99_and_a_c_host_calls_the_library(ndlib, tmp_path):
    src = tmp_path / "host.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "host"
    libdir = os.path.dirname(runtime.LIB_PATH)
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", INCLUDE, str(src), "-o", str(exe),
           "-L", libdir, "-l:libnd_march.so", f"-Wl,-rpath,{libdir}", "-Wl,--allow-shlib-undefined"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    words = run.stdout.split()
    assert words[0] == "ND_ERR_TIMEOUT" and words[2] == "Power" and float(words[3]) == 8.0
    assert int(words[1]) == runtime.formula_count()
