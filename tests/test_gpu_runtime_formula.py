"""A formula compiled at run time (nd_formula_register) on the GPU.  The edited copy of
the package's Mandelbulb differs from the built-in one only in a @param default, so
its kernels are the same code: its DE at points and its forward march must equal the
built-in formula's bit for bit, and with Bailout = 2 its FP64 DE must match the golden
values of the reference's own Mandelbulb (tests/golden/de_reference_fp64.json, made
from the reference's formula code) as the built-in one does."""

import json
import os

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads
from tests.test_runtime_formula import edited_source

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "de_reference_fp64.json")


def test_runtime_formula_matches_the_built_in_and_the_golden_values(ctx):
    fid = runtime.register_formula(edited_source())
    builtin = runtime.find_formula("mandelbulb_bailout")
    assert fid != builtin
    with open(GOLDEN) as fh:
        entries = json.load(fh)["formulas"]["mandelbrot"]
    worst = 0.0
    for e in entries:
        power, iters = e["params"][0], e["params"][1]
        pts = np.asarray(e["points"])
        va = abi.make_view(fid, 1, 1, (0.0, 0.0, -3.0), params=[power, iters, 2.0])
        vb = abi.make_view(builtin, 1, 1, (0.0, 0.0, -3.0), params=[power, iters, 2.0])
        for prec in (32, 64):
            da, ta, ia = ctx.de_points(va, pts, prec)
            db, tb, ib = ctx.de_points(vb, pts, prec)
            np.testing.assert_array_equal(da, db)
            np.testing.assert_array_equal(ta, tb)
            np.testing.assert_array_equal(ia, ib)
        d64, _, _ = ctx.de_points(va, pts, 64)
        ref = np.asarray(e["de"])
        worst = max(worst, float((np.abs(d64 - ref) / np.maximum(np.abs(ref), 1e-30)).max()))
    print("runtime-compiled Mandelbulb (Bailout 2) vs reference Mandelbulb, fp64 max rel", worst)
    assert worst <= 1e-9

    # a forward march of views of it: the built-in formula's bits
    views = []
    for formula in (fid, builtin):
        v, _ = workloads.mandelbulb_512(lambda name: formula, power=8.0, size=96)
        views.append(v)
    outs = []
    for v in views:
        g = runtime.GBuffer.allocate(abi.rays_of(v))
        ctx.forward([v], g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
        outs.append(g.numpy())
    for k in ("depth64", "steps", "evals", "normal", "shade", "trap", "iters"):
        np.testing.assert_array_equal(outs[0][k], outs[1][k], err_msg=k)
    assert (outs[0]["normal"][:, 3] > 0.5).any()
