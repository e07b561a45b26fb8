"""Scene files rendered on the GPU: a .dream scene loaded by nd_scene_file_load and
marched by nd_march_forward_scenes against the oracle's scene march of the same
descriptors (boundary-case policy; depth p99 <= 1e-4, normal p99 <= 2 degrees over
stable short rays both hit).  One scene is the fixture tests/golden/two_fractals.dream
(Mandelbulb and a Mandelbox with a Menger mixin); the other stands fractals on and
beside primitives (a flat box floor, a sphere, a Menger sponge), the way the
reference's own bench scenes are built."""

import json
import os

import numpy as np

import pytest

from numericdream_b200 import runtime, workloads
from tests.parity_util import compare, policy_check

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _render_and_check(ctx, view, scene, min_hits=100):
    from oracle import pyoracle

    g = runtime.GBuffer.allocate(workloads.rays([view]))
    if scene is None:
        ctx.forward([view], g)
    else:
        ctx.forward_scenes([view], [0], [scene], g)
    st = ctx.stats()
    assert st.timeouts == 0
    gpu = g.numpy()
    if scene is None:
        unstable, base = pyoracle.unstable_rays(view, runtime.formula_name(view.formula))
    else:
        unstable, base = pyoracle.unstable_scene_rays(view, scene, runtime.formula_name)
    pol = policy_check(gpu, base, unstable)
    strict = pol.pop("strict_mask")
    print("policy:", pol)
    assert pol["ok"], pol
    c = compare(gpu, base, mask=strict)
    print("vs oracle f64 (stable short rays):", c)
    assert c["hits_ref"] >= min_hits
    assert c["depth_rel_p99"] <= 1e-4
    assert c["normal_deg_p99"] <= 2.0


def test_fixture_scene_file(ctx):
    view, scene = runtime.load_scene_file(os.path.join(HERE, "golden", "two_fractals.dream"), 128, 72)
    assert scene is not None
    _render_and_check(ctx, view, scene)


def test_fractal_on_primitives(ctx):
    def inst(path, offset, scale, params=(), **kw):
        d = {"offset": dict(zip("xyz", offset)), "scale": dict(zip("xyz", scale)),
             "rotation": {"x": 0, "y": 0, "z": 0}, "step_safety": 1.0, "combine_mode": "hard_union",
             "blend_k": 0.5, "formula": {"path": path, "params": [{"name": n, "value": v} for n, v in params]},
             "mixins": [], "hybrid_base_iters": 1, "hybrid_total_iters": 8, "colors": []}
        d.update(kw)
        return d

    doc = {"version": 12,
           "camera": {"position": {"x": 0.3, "y": 0.7, "z": 4.0}, "forward": {"x": -0.07, "y": -0.19, "z": -0.979},
                      "up": {"x": -0.014, "y": 0.982, "z": -0.19}},
           "render_settings": {"max_steps": 256, "max_dist": 24},
           "export_width": 112, "export_height": 64,
           "instances": [inst("", (0, 0, 0), (1, 1, 1), rotation={"x": 20, "y": 30, "z": 0}),
                         inst("formulas/cube_primitive.wgsl", (0, -1.35, 0), (6, 0.1, 6)),
                         inst("formulas/menger3_ifs.wgsl", (2.1, -0.45, -1.2), (0.75, 0.75, 0.75)),
                         inst("formulas/sphere_primitive.wgsl", (-1.75, -0.8, 0.7), (1, 1, 1), [("Radius", 0.45)])],
           "lights": [], "fog_emitters": []}
    view, scene = runtime.load_scene_file(json.dumps(doc))
    assert scene is not None and scene.instance_count == 4
    _render_and_check(ctx, view, scene, min_hits=1000)


def test_render_scene_file_to_an_image(ctx, tmp_path):
    """The fixture scene file to a colour image (geometry + lite shading with its
    colour stops and lights) against the oracle's lite shading of the same hits."""
    from numericdream_b200 import abi
    from numericdream_b200.render import render_scene_file, write_ppm
    from oracle import pyoracle

    path = os.path.join(HERE, "golden", "two_fractals.dream")
    img, g = render_scene_file(ctx, path, 160, 90)
    assert img.shape == (90, 160, 4)
    hit = g["normal"][:, 3] > 0.5
    np.testing.assert_array_equal(img.reshape(-1, 4)[:, 3], hit.astype(np.float32))
    view, scene = runtime.load_scene_file(path, 160, 90)
    lite = runtime.load_scene_file_lite(path, 0)
    colors = []
    for i in range(scene.instance_count):
        c = runtime.load_scene_file_lite(path, i)
        stops = sorted(((tuple(s.color), s.position, s.glossiness, s.ior) for s in c.colors[:c.color_count]),
                       key=lambda s: s[1])
        colors.append(abi.make_lite(stops))
    ref = pyoracle.shade_lite_scene(view, scene, runtime.formula_name, lite, colors, g, precision=32)
    err = np.abs(img.reshape(-1, 4)[hit, :3] - ref[hit, :3]).max(axis=1)
    assert hit.sum() > 500 and (err <= 2e-3).mean() >= 0.99
    out = tmp_path / "scene.ppm"
    write_ppm(str(out), img)
    assert out.read_bytes().startswith(b"P6 160 90 255\n") and out.stat().st_size == 14 + 160 * 90 * 3


def test_fractal_renderer_render_to_image(ctx):
    from numericdream_b200.runtime import FractalRenderer

    r = FractalRenderer(0)
    try:
        data = r.render_to_image(os.path.join(HERE, "golden", "two_fractals.dream"), 64, 36)
    finally:
        r.ctx.close()
    img = np.frombuffer(data, np.uint8).reshape(36, 64, 4)
    assert (img[..., 3] == 255).all() and img[..., :3].std() > 1.0
