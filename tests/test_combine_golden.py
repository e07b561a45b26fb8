"""The instance combine modes (combine_de, template.wgsl:1708-1730, and the smooth
operators smin ... smix, :1653-1706) against the reference's own code run in f32
(tests/golden/combine_reference_f32.json, written by oracle/_ref): the oracle's
restatement and the CUDA library's combine_de and combine_weight (its header
compiled for the host with g++, same source the kernels use) give the same bits,
distance and material weight."""

import json
import os
import subprocess
import tempfile

import numpy as np

from oracle import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden", "combine_reference_f32.json")

PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include "nd_rayprog.h"
int main() {
  int mode; float d, di, k;
  while (std::scanf("%d %a %a %a", &mode, &d, &di, &k) == 4)
    std::printf("%a %a\n", double(nd::combine_de<float>(mode, d, di, k)),
                double(nd::combine_weight<float>(mode, d, di, k)));
  return 0;
}
"""


def _golden(weight=False):
    with open(GOLDEN) as fh:
        g = json.load(fh)
    return (np.array(g["mode"], np.int32), np.array(g["d"], np.float32), np.array(g["di"], np.float32),
            np.array(g["k"], np.float32), np.array(g["weight" if weight else "de"], np.float32))


def test_oracle_combine_matches_the_reference():
    mode, d, di, k, want = _golden()
    assert sorted(set(mode.tolist())) == list(range(7))
    got = pyoracle.combine(mode, d, di, k)
    np.testing.assert_array_equal(got, want)


def test_oracle_combine_weight_matches_the_reference():
    mode, d, di, k, want = _golden(weight=True)
    np.testing.assert_array_equal(pyoracle.combine_weight(mode, d, di, k), want)


def test_cuda_combine_de_matches_the_reference():
    mode, d, di, k, want = _golden()
    _, _, _, _, want_w = _golden(weight=True)
    with tempfile.TemporaryDirectory() as tmp:
        cpp, exe = os.path.join(tmp, "c.cpp"), os.path.join(tmp, "c")
        with open(cpp, "w") as fh:
            fh.write(PROGRAM)
        subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I",
                        os.path.join(ROOT, "numericdream_b200", "csrc"), cpp, "-o", exe], check=True)
        inp = "\n".join(f"{m} {float(a).hex()} {float(b).hex()} {float(c).hex()}" for m, a, b, c in zip(mode, d, di, k))
        res = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split()
    got = np.array([float.fromhex(x) for x in res], np.float32).reshape(-1, 2)
    np.testing.assert_array_equal(got[:, 0], want)
    np.testing.assert_array_equal(got[:, 1], want_w)
