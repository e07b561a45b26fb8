"""GPU lite shading (nd_shade_lite: shade_lite, template.wgsl:4424-4444) against the
oracle's lite shading of the same forward outputs: every channel within 2e-3 on
99 % of the hits (FP32 DE for the ambient-occlusion taps, f32 shading arithmetic
on both sides of the reference's formulas), misses the background exactly."""

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu

STOPS = [((0.05, 0.05, 0.22), 0.0, 0.2, 1.3), ((0.85, 0.35, 0.08), 0.5, 0.5, 1.5), ((1.0, 0.95, 0.82), 1.0, 0.8, 1.7)]
LIGHTS = [(abi.ND_LIGHT_GLOBAL, (0.4, 0.8, -0.45), (1.0, 0.95, 0.9), 1.2),
          (abi.ND_LIGHT_POINT, (2.0, 2.5, -3.0), (0.6, 0.7, 1.0), 6.0)]


def _check(ctx, views, lites):
    from oracle import pyoracle

    g = runtime.GBuffer.allocate(workloads.rays(views))
    ctx.forward(views, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    rgba = ctx.shade_lite(views, lites, g).cpu().numpy()
    out = g.numpy()
    off = 0
    for v, lite in zip(views, lites):
        n = workloads.rays([v])
        sl = {k: a[off:off + n] for k, a in out.items()}
        ref = pyoracle.shade_lite(v, runtime.formula_name(v.formula), lite, sl, precision=32)
        got = rgba[off:off + n]
        hit = sl["normal"][:, 3] > 0.5
        np.testing.assert_array_equal(got[:, 3], hit.astype(np.float32))
        np.testing.assert_array_equal(got[~hit, :3], np.tile(np.array(lite.background, np.float32), ((~hit).sum(), 1)))
        err = np.abs(got[hit, :3] - ref[hit, :3]).max(axis=1)
        print(runtime.formula_name(v.formula), "hits", hit.sum(), "max err", err.max(initial=0), "p99",
              np.percentile(err, 99) if hit.any() else 0)
        if hit.any():
            assert (err <= 2e-3).mean() >= 0.99
            assert np.ptp(got[hit, 0]) > 0.05  # the strip and the lights vary the colour
        off += n


def test_lite_shading_single_views(ctx):
    for name, prm, cam, trap in ((workloads.MANDELBOX, workloads.mandelbox_params(-1.5, 12), (0.3, 0.6, -4.2),
                                  {"shape": abi.ND_TRAP_BOX, "span": 1.5}),
                                 (workloads.MANDELBULB, workloads.mandelbulb_params(8.0, 10), (0.5, 0.9, -2.6),
                                  {"shape": abi.ND_TRAP_SPHERE, "radius": 1.0, "span": 0.8, "repeat": 2})):
        v = abi.make_view(runtime.find_formula(name), 96, 80, cam, fov_y_deg=60.0, params=prm, max_steps=256,
                          trap=trap)
        _check(ctx, [v], [abi.make_lite(STOPS, LIGHTS)])


def test_lite_shading_batched_and_unsorted_stops(ctx):
    views = workloads.batched_64(runtime.find_formula, nviews=6, max_side=128, seed=3)
    lites = []
    for i in range(len(views)):
        stops = STOPS if i % 2 == 0 else list(reversed(STOPS))  # the library sorts them
        lites.append(abi.make_lite(stops, LIGHTS[: 1 + i % 2], ambient_occlusion=i % 3 != 2, specular=i % 2 == 0))
    _check(ctx, views, [abi.make_lite(sorted(STOPS, key=lambda s: s[1]), LIGHTS[: 1 + i % 2],
                                      ambient_occlusion=i % 3 != 2, specular=i % 2 == 0) for i in range(len(views))])
    # the reversed stop lists give the same pixels as the sorted ones
    g = runtime.GBuffer.allocate(workloads.rays(views))
    ctx.forward(views, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    a = ctx.shade_lite(views, lites, g).cpu().numpy()
    b = ctx.shade_lite(views, [abi.make_lite(sorted(STOPS, key=lambda s: s[1]), LIGHTS[: 1 + i % 2],
                                             ambient_occlusion=i % 3 != 2, specular=i % 2 == 0)
                               for i in range(len(views))], g).cpu().numpy()
    np.testing.assert_array_equal(a, b)


def test_lite_refusals(ctx):
    v = abi.make_view(runtime.find_formula(workloads.MANDELBOX), 16, 16, (0.3, 0.6, -4.2),
                      params=workloads.mandelbox_params(-1.5, 12))
    g = runtime.GBuffer.allocate(256)
    ctx.forward([v], g)
    bad = abi.make_lite(STOPS, LIGHTS)
    bad.lights[0].type = 2  # ray lights are not in this pass
    with pytest.raises(runtime.NDError) as e:
        ctx.shade_lite([v], [bad], g)
    assert e.value.status == abi.ND_ERR_UNSUPPORTED
    g.trap = None
    with pytest.raises(runtime.NDError) as e:
        ctx.shade_lite([v], [abi.make_lite(STOPS, LIGHTS)], g)
    assert e.value.status == abi.ND_ERR_INVALID


def test_lite_shading_of_a_scene(ctx):
    """A Mandelbulb on a box floor beside a sphere, each instance with its own colour
    strip, against the oracle's hit_material blend."""
    from oracle import pyoracle

    fid = runtime.find_formula
    bulb = abi.make_instance(fid(workloads.MANDELBULB), params=workloads.mandelbulb_params(8.0, 8),
                             trap={"shape": abi.ND_TRAP_SPHERE, "radius": 0.8, "span": 1.0})
    floor = abi.make_instance(fid("cube_primitive"), params=[1.0], offset=(0.0, -1.35, 0.0), scale=(6.0, 0.1, 6.0),
                              combine_mode=abi.ND_COMBINE_SMOOTH_MIN, blend_k=0.3)
    ball = abi.make_instance(fid("sphere_primitive"), params=[0.45], offset=(-1.4, -0.8, 0.6),
                             trap={"shape": abi.ND_TRAP_POINT, "span": 2.0, "repeat": 1})
    scene = abi.make_scene([bulb, floor, ball])
    v = abi.make_view(fid(workloads.MANDELBULB), 96, 72, (0.3, 0.7, -3.6), fov_y_deg=60.0, max_steps=256)
    colors = [abi.make_lite(STOPS), abi.make_lite([((0.3, 0.3, 0.3), 0.0, 0.1, 1.2)]),
              abi.make_lite(list(reversed(STOPS)))]
    lite = abi.make_lite([], LIGHTS)
    g = runtime.GBuffer.allocate(workloads.rays([v]))
    ctx.forward_scenes([v], [0], [scene], g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    rgba = ctx.shade_lite_scenes([v], [0], [scene], [lite], [colors], g).cpu().numpy()
    out = g.numpy()
    sorted_colors = [abi.make_lite(sorted(STOPS, key=lambda s: s[1])), colors[1],
                     abi.make_lite(sorted(STOPS, key=lambda s: s[1]))]
    ref = pyoracle.shade_lite_scene(v, scene, runtime.formula_name, lite, sorted_colors, out, precision=32)
    hit = out["normal"][:, 3] > 0.5
    assert hit.sum() > 1000
    err = np.abs(rgba[hit, :3] - ref[hit, :3]).max(axis=1)
    print("scene lite: hits", hit.sum(), "max err", err.max(), "p99", np.percentile(err, 99))
    assert (err <= 2e-3).mean() >= 0.99
    # the three materials all show up
    assert np.ptp(rgba[hit, 2]) > 0.1
