"""Error bounds of the polynomial f32 acos / atan2 (nd_wgsl.h) that the fast-math
device build uses instead of acosf / atan2f: compiled here for the host with g++
(same source, f32 arithmetic with FMA) and compared with double-precision libm on
dense grids and on the special cases."""

import os
import subprocess
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "numericdream_b200", "csrc")

PROGRAM = r"""
#include <cmath>
#include <cstdio>
#include "nd_wgsl.h"
int main() {
  // acos on [-1, 1]
  double worst_acos = 0.0;
  for (int i = 0; i <= 2000000; ++i) {
    const float x = -1.0f + 2.0f * float(i) / 2000000.0f;
    const double e = std::fabs(double(ndw::nd_acos_poly(x)) - std::acos(double(x)));
    if (e > worst_acos) worst_acos = e;
  }
  // atan2 on a polar grid of radii 1e-30 .. 1e30 and all angles
  double worst_atan2 = 0.0;
  for (int k = -30; k <= 30; k += 3) {
    const double rad = std::pow(10.0, k);
    for (int i = 0; i < 200000; ++i) {
      const double ang = -3.14159265358979 + 6.28318530717959 * (i + 0.5) / 200000.0;
      const float y = float(rad * std::sin(ang)), x = float(rad * std::cos(ang));
      const double e = std::fabs(double(ndw::nd_atan2_poly(y, x)) - std::atan2(double(y), double(x)));
      if (e > worst_atan2) worst_atan2 = e;
    }
  }
  std::printf("%.9g %.9g\n", worst_acos, worst_atan2);
  const float pz = 0.0f, nz = -0.0f, inf = INFINITY;
  const float cases[][2] = {{pz, pz}, {pz, nz}, {nz, pz}, {nz, nz}, {1.0f, pz}, {-1.0f, pz}, {pz, -1.0f},
                            {nz, -1.0f}, {inf, inf}, {-inf, inf}, {inf, -inf}, {2.0f, inf}, {2.0f, -inf}};
  for (const auto& c : cases) std::printf("%.9g %.9g\n", double(ndw::nd_atan2_poly(c[0], c[1])), std::atan2(double(c[0]), double(c[1])));
  std::printf("%.9g %.9g %.9g\n", double(ndw::nd_acos_poly(1.0f)), double(ndw::nd_acos_poly(-1.0f)),
              double(ndw::nd_acos_poly(0.0f)));
  std::printf("%d %d\n", int(std::isnan(ndw::nd_acos_poly(NAN))), int(std::isnan(ndw::nd_atan2_poly(NAN, 1.0f))));
  return 0;
}
"""


def test_polynomial_acos_atan2_error_bounds():
    with tempfile.TemporaryDirectory() as d:
        cpp = os.path.join(d, "m.cpp")
        exe = os.path.join(d, "m")
        with open(cpp, "w") as fh:
            fh.write(PROGRAM)
        subprocess.run(["g++", "-std=c++17", "-O2", "-I", CSRC, cpp, "-o", exe], check=True)
        lines = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    worst_acos, worst_atan2 = map(float, lines[0].split())
    print("max |error|: acos", worst_acos, "atan2", worst_atan2)
    # a few f32 ulp of pi (2.4e-7); the fits themselves are within 2.2e-8
    assert worst_acos <= 5e-7
    assert worst_atan2 <= 5e-7
    for line in lines[1:14]:
        got, want = map(float, line.split())
        assert abs(got - want) <= 5e-7 and np.copysign(1.0, got) == np.copysign(1.0, want), line
    a1, am1, a0 = map(float, lines[14].split())
    assert a1 == 0.0 and abs(am1 - np.pi) <= 3e-7 and abs(a0 - np.pi / 2) <= 3e-7
    assert lines[15].split() == ["1", "1"]
