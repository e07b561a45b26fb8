"""CUDA DE of every formula against the reference's own formula code (FP64 golden
values from tests/golden, computed by the reference WGSL translated and compiled on
the host), through the C ABI's nd_de_points."""

import json
import os

import numpy as np
import pytest

from numericdream_b200 import abi, runtime

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "de_reference_fp64.json")


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-9)


def test_gpu_de_matches_reference_golden(ctx):
    with open(GOLDEN) as fh:
        golden = json.load(fh)["formulas"]
    names = set(runtime.formula_names())
    worst64, worst32 = {}, {}
    for name, entries in golden.items():
        assert name in names, f"{name} missing from the build"
        fid = runtime.find_formula(name)
        r64, r32 = [], []
        for e in entries:
            v = abi.make_view(fid, 1, 1, (0.0, 0.0, -3.0), params=e["params"])
            pts = np.asarray(e["points"])
            want = np.asarray(e["de"])
            d64, _, _ = ctx.de_points(v, pts, 64)
            d32, _, _ = ctx.de_points(v, pts, 32)
            r64.append(_rel(d64, want))
            r32.append(_rel(d32, want))
        r64 = np.concatenate(r64)
        r32 = np.concatenate(r32)
        worst64[name] = (float(np.median(r64)), float(r64.max()))
        worst32[name] = (float(np.median(r32)), float(np.percentile(r32, 90)))
    for name in sorted(golden):
        print(f"{name:32s} fp64 median {worst64[name][0]:.2e} max {worst64[name][1]:.2e} | "
              f"fp32 median {worst32[name][0]:.2e} p90 {worst32[name][1]:.2e}")
    # FP64 on the GPU follows the reference code to rounding (FMA contraction only)
    assert all(m <= 1e-9 for m, _ in worst64.values()), worst64
    # the FP32 fast-math DE stays within FP32 noise on the typical point
    assert all(m <= 1e-3 for m, _ in worst32.values()), worst32


def test_mandelbulb_bailout_at_2_is_the_reference_mandelbulb(ctx):
    """The package's mandelbulb_bailout formula with Bailout = 2 against the golden
    values of the reference's built-in Mandelbulb (same power and iterations)."""
    with open(GOLDEN) as fh:
        entries = json.load(fh)["formulas"]["mandelbrot"]
    fid = runtime.find_formula("mandelbulb_bailout")
    worst = 0.0
    for e in entries:
        power, iters = e["params"][0], e["params"][1]
        v = abi.make_view(fid, 1, 1, (0.0, 0.0, -3.0), params=[power, iters, 2.0])
        d64, _, _ = ctx.de_points(v, np.asarray(e["points"]), 64)
        worst = max(worst, float(_rel(d64, np.asarray(e["de"])).max()))
    print("mandelbulb_bailout(2) vs reference Mandelbulb, fp64 max rel", worst)
    assert worst <= 1e-9


MARCH_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "march_reference_fp64.json")


@pytest.mark.parametrize("kernel", [abi.ND_KERNEL_PERSISTENT, abi.ND_KERNEL_PLAIN])
def test_gpu_march_matches_the_reference_march(ctx, kernel):
    """The CUDA march with an FP64 DE against the reference's own march code run in
    FP64 (tests/golden/march_reference_fp64.json: march_to, bisection, verify and
    high-quality modes, tetrahedral normals): the hit decisions and probe steps agree
    but for rays the last bits of the DE decide (the GPU's FP64 DE contracts into
    FMAs), the hit distance to 1e-9, the normal to 0.05 degrees (summed in f32)."""
    with open(MARCH_GOLDEN) as fh:
        cases = json.load(fh)["cases"]
    for c in cases:
        v = abi.make_view(runtime.find_formula(c["formula"]), 16, 16, tuple(c["camera"]), fov_y_deg=60.0,
                          params=c["params"], max_steps=256, **c["mode"])
        g = runtime.GBuffer.allocate(256)
        ctx.forward([v], g, runtime.make_opts(kernel=kernel, de_precision=64))
        o = g.numpy()
        hit = np.array(c["hit"]) == 1
        gh = o["normal"][:, 3] > 0.5
        what = f"{c['formula']} {c['mode']}"
        assert (gh != hit).sum() <= 1, what
        assert (o["steps"] != np.array(c["steps"])).sum() <= 2, what
        both = gh & hit
        t = np.array(c["t"])
        if both.any():
            rel = np.abs(o["depth64"][both] - t[both]) / t[both]
            # a ray whose last DE bits flip a probe or bisection decision ends within
            # eps(t) of the reference's hit; the others agree to the FP64 DE's rounding
            assert rel.max() <= 1e-4, (what, rel.max())
            assert (rel <= 1e-9).mean() >= 0.95, (what, np.sort(rel)[-5:])
            ang = np.degrees(np.arccos(np.clip((o["normal"][both, :3] * np.array(c["normal"])[both]).sum(1), -1, 1)))
            # the normal sums its taps in f32 (as the reference does), so it carries
            # f32 cancellation even with an FP64 DE: a few hundredths of a degree
            assert np.percentile(ang, 99) <= 0.05, what


TRAP_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "trap_reference_fp64.json")


def test_gpu_trap_matches_the_reference_wrapper(ctx):
    """The CUDA formula wrapper's DE and orbit trap (nd_de_points, FP64 and FP32) against
    the reference's generated wrapper with its trap functions run in FP64."""
    from tests.test_oracle import trap_desc

    with open(TRAP_GOLDEN) as fh:
        cases = json.load(fh)["cases"]
    worst64 = worst32 = 0.0
    for c in cases:
        v = abi.make_view(runtime.find_formula(c["formula"]), 1, 1, (0.0, 0.0, -3.0), params=c["params"])
        v.trap = trap_desc(c["trap"])
        pts = np.asarray(c["points"])
        d64, t64, _ = ctx.de_points(v, pts, 64)
        d32, t32, _ = ctx.de_points(v, pts, 32)
        want = np.asarray(c["trap_value"])
        worst64 = max(worst64, float(np.max(_rel(t64, want))))
        worst32 = max(worst32, float(np.median(_rel(t32, want))))
        np.testing.assert_allclose(d64, c["de"], rtol=1e-9, atol=1e-12)
    print("trap: fp64 max rel", worst64, "fp32 worst median rel", worst32)
    # FP64 to rounding (the GPU contracts into FMAs along the iterations)
    assert worst64 <= 1e-8
    assert worst32 <= 1e-3


SHADE_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "shade_reference_fp64.json")


def test_gpu_shade_and_shadow_match_the_reference(ctx):
    """The CUDA Lambert level and shadow visibility (FP64 DE) against the reference's
    simple_geometry and visibility_march run in FP64."""
    with open(SHADE_GOLDEN) as fh:
        cases = json.load(fh)["cases"]
    for c in cases:
        kw = dict(shadow=1, light_dir=(0.4, 0.8, -0.45)) if c["shadow"] else {}
        v = abi.make_view(runtime.find_formula(c["formula"]), 16, 16, tuple(c["camera"]), fov_y_deg=90.0,
                          params=c["params"], max_steps=256, **kw)
        g = runtime.GBuffer.allocate(256)
        ctx.forward([v], g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=64))
        o = g.numpy()
        hit = (np.array(c["hit"]) == 1) & (o["normal"][:, 3] > 0.5)
        if c["shadow"]:
            dv = np.abs(o["shadow"][hit] - np.array(c["visibility"])[hit])
            share = 0.8 if c["formula"] == "pseudokleinian_kleinian" else 0.97
            assert (dv <= 1e-4).mean() >= share, (c["formula"], (dv <= 1e-4).mean())
        else:
            ds = np.abs(o["shade"][hit] - np.array(c["shade"])[hit])
            assert np.percentile(ds, 99) <= 1e-4, (c["formula"], ds.max())
