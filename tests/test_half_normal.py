"""The RGBA16F normal output's float-to-half conversion (the host build of the ray
program's half_bits, used where no GPU is) against numpy's IEEE binary16 rounding
(round to nearest even) over normals, subnormals, overflow, infinities and NaN."""

import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <cstring>
#include "nd_rayprog.h"
int main() {
  unsigned u;
  while (std::scanf("%x", &u) == 1) {
    float x;
    std::memcpy(&x, &u, 4);
    std::printf("%u\n", unsigned(nd::half_bits(x)));
  }
  return 0;
}
"""


def test_half_bits_rounds_like_ieee():
    rng = np.random.default_rng(3)
    xs = np.concatenate([
        rng.uniform(-1.0, 1.0, 20000), rng.normal(0, 1e-5, 5000), rng.normal(0, 1e4, 3000),
        np.array([0.0, -0.0, 65504.0, 65519.99, 65520.0, 1e9, -1e9, np.inf, -np.inf, 2.0 ** -24, 2.0 ** -25,
                  3 * 2.0 ** -26, 2.0 ** -14, 2.0 ** -14 * (1 - 2.0 ** -12), 1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11,
                  np.nan])])
    xs = xs.astype(np.float32)
    with tempfile.TemporaryDirectory() as d:
        cpp, exe = os.path.join(d, "h.cpp"), os.path.join(d, "h")
        with open(cpp, "w") as fh:
            fh.write(PROGRAM)
        subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "numericdream_b200", "csrc"), cpp, "-o",
                        exe], check=True)
        inp = "\n".join(f"{int(b):08x}" for b in xs.view(np.uint32))
        out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split()
    got = np.array([int(x) for x in out], np.uint16)
    with np.errstate(over="ignore"):
        want = xs.astype(np.float16).view(np.uint16)
    np.testing.assert_array_equal(got, want)
