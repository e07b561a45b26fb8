"""Lite shading (shade_lite, template.wgsl:4424-4444): the oracle's ambient occlusion,
colour-strip position and Fresnel term against the reference's calc_ao,
orbit_trap_to_strip and fresnel_schlick (tests/golden/lite_reference.json, written
by oracle/_ref), and the oracle's colour strip and light terms against closed forms."""

import json
import os

import numpy as np

from numericdream_b200 import abi
from oracle import pyoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lite_reference.json")


def _golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


def test_ao_matches_the_reference():
    g = _golden()["ao"]
    assert len(g) == 6
    for c in g:
        v = abi.make_view(0, 16, 16, tuple(c["camera"]), fov_y_deg=60.0, params=c["params"], max_steps=256)
        got = pyoracle.ao(v, c["formula"], np.array(c["pos"]), np.array(c["normal"]), np.array(c["t"]), 64)
        np.testing.assert_allclose(got, c["ao"], rtol=1e-12, atol=1e-12, err_msg=c["formula"])
        assert len(c["ao"]) > 0 and (np.array(c["ao"]) < 1).any() or c["formula"] in ("sphere_primitive",
                                                                                      "cube_primitive")


def test_strip_and_fresnel_match_the_reference():
    g = _golden()["strip_fresnel"]
    st, fr = pyoracle.strip_fresnel(g["span_offset_repeat"], g["v"], g["cos"], g["ior"])
    np.testing.assert_array_equal(st, np.array(g["strip"], np.float32))
    np.testing.assert_array_equal(fr, np.array(g["fresnel"], np.float32))


def test_lite_colour_strip_and_lights_closed_form():
    # a sphere of radius 1 with a point trap at its centre: the trap of a hit is the
    # distance of the hit point to the centre, 1; span 2 puts it at strip 0.5, midway
    # between a red stop at 0 and a blue stop at 1
    v = abi.make_view(0, 17, 17, (0.0, 0.0, -3.0), fov_y_deg=40.0, params=[1.0], max_steps=256,
                      trap={"shape": abi.ND_TRAP_POINT, "mode": abi.ND_TRAP_LAST, "span": 2.0})
    o = pyoracle.render(v, "sphere_primitive", 64)
    c = 8 * 17 + 8
    assert o["normal"][c, 3] == 1.0
    np.testing.assert_allclose(o["trap"][c], 1.0, atol=1e-5)
    lite = abi.make_lite(colors=[((1, 0, 0), 0.0, 0.0, 1.0), ((0, 0, 1), 1.0, 0.0, 1.0)],
                         lights=[(abi.ND_LIGHT_GLOBAL, (0.0, 0.0, -1.0), (1, 1, 1), 2.0)], ambient_occlusion=False,
                         specular=False)
    rgba = pyoracle.shade_lite(v, "sphere_primitive", lite, o)
    # centre ray: normal (0, 0, -1), light along the normal (ndotl 1), ior 1 (no
    # Fresnel), glossiness 0: colour (0.5, 0, 0.5) x (0.15 ambient + 2)
    np.testing.assert_allclose(rgba[c, :3], [0.5 * 2.15, 0.0, 0.5 * 2.15], atol=1e-4)
    assert rgba[c, 3] == 1.0
    miss = np.where(o["normal"][:, 3] < 0.5)[0][0]
    np.testing.assert_allclose(rgba[miss], list(lite.background) + [0.0], atol=1e-7)
    # a point light at distance r falls off as 1 / r^2
    lite.lights[0].type = abi.ND_LIGHT_POINT
    lite.lights[0].position_or_direction[:] = [0.0, 0.0, -3.0]
    rgba = pyoracle.shade_lite(v, "sphere_primitive", lite, o)
    r = 3.0 - o["depth64"][c] * 0.0 - 1.0  # the hit is at z = -1, the light at z = -3
    np.testing.assert_allclose(rgba[c, 0], 0.5 * (0.15 + 2.0 / r ** 2), rtol=1e-4)
