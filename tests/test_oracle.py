"""The CPU oracle, pinned against the reference's own formula code (golden DE values
from oracle/_ref, committed in tests/golden) and against closed-form answers."""

import json
import math
import os

import numpy as np
import pytest

from numericdream_b200 import abi
from oracle import pyoracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "de_reference_fp64.json")
ORACLE_FORMULAS = ["mandelbrot", "amazingbox_box", "menger3_ifs", "pseudokleinian_kleinian", "sphere_primitive",
                   "cube_primitive"]


def _golden():
    with open(GOLDEN) as fh:
        return json.load(fh)["formulas"]


@pytest.mark.parametrize("name", ORACLE_FORMULAS)
def test_oracle_de_matches_reference_golden(name):
    g = _golden()[name]
    for entry in g:
        pts = np.asarray(entry["points"])
        want = np.asarray(entry["de"])
        got, _, _ = pyoracle.de(name, entry["params"], pts, 64)
        rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
        assert rel.max() <= 1e-12, (name, entry["params"][:6], rel.max())


def test_golden_covers_every_formula():
    g = _golden()
    assert len(g) >= 54
    for name in ORACLE_FORMULAS:
        assert name in g


def _view(formula_name, size, cam_z, params, **kw):
    fid = 0  # the oracle takes the formula by name; the id is not used
    return abi.make_view(fid, size, size, (0.0, 0.0, cam_z), fov_y_deg=60.0, params=params, **kw)


def test_sphere_known_answer():
    # camera on the -z axis looking at a sphere of radius R at the origin: the
    # centre ray hits at t = |cam| - R, normal -z; every hit lies on the sphere
    R, cz = 1.25, -3.0
    v = _view("sphere_primitive", 65, cz, [R], eps_coef=1e-5, eps_floor=0.0, max_steps=512)
    o = pyoracle.render(v, "sphere_primitive", 64)
    c = 32 * 65 + 32
    assert o["normal"][c, 3] == 1.0
    assert abs(o["depth64"][c] - (abs(cz) - R)) <= 1e-5 * (abs(cz) - R)
    np.testing.assert_allclose(o["normal"][c, :3], [0.0, 0.0, -1.0], atol=1e-6)
    # all hits on the surface: |org + dir t| = R within eps(t)
    hits = np.where(o["normal"][:, 3] > 0.5)[0]
    assert len(hits) > 100
    # closed-form hit count: rays whose distance to the origin is < R
    tan30 = math.tan(math.radians(30.0))
    n_expect = 0
    for idx in range(65 * 65):
        px, py = idx % 65, idx // 65
        ux = (2.0 * (px + 0.5) / 65 - 1.0) * tan30
        uy = (2.0 * (py + 0.5) / 65 - 1.0) * tan30
        d = np.array([ux, uy, 1.0]) / math.sqrt(ux * ux + uy * uy + 1.0)
        o_ = np.array([0.0, 0.0, cz])
        b = o_ @ d
        disc = b * b - (o_ @ o_ - R * R)
        if disc > 1e-9:
            n_expect += 1
            t = -b - math.sqrt(disc)
            if o["normal"][idx, 3] > 0.5:
                # sphere tracing an exact SDF never overshoots: the hit is in front
                # of the true intersection and within eps(t) of the surface
                got = o["depth64"][idx]
                eps = 1e-5 * got
                assert got <= t + 1e-12
                r = np.linalg.norm(o_ + d * got)
                assert -1e-12 <= r - R < eps, (idx, r - R, eps)
                # and short of it by at most eps / cos(incidence), cos = sqrt(disc) / R
                assert got >= t - eps * R / math.sqrt(disc) - 1e-9, (idx, got, t)
    assert abs(len(hits) - n_expect) <= 4


def test_cube_known_answer():
    s, cz = 0.7, -2.5
    v = _view("cube_primitive", 33, cz, [s], eps_coef=1e-5, eps_floor=0.0, max_steps=512)
    o = pyoracle.render(v, "cube_primitive", 64)
    c = 16 * 33 + 16
    assert abs(o["depth64"][c] - (abs(cz) - s)) <= 1e-5
    np.testing.assert_allclose(o["normal"][c, :3], [0.0, 0.0, -1.0], atol=1e-5)


def test_fp32_oracle_close_to_fp64():
    v = _view("mandelbrot", 48, -2.5, [8.0, 12.0], eps_coef=1e-4, eps_floor=0.0)
    a = pyoracle.render(v, "mandelbrot", 32)
    b = pyoracle.render(v, "mandelbrot", 64)
    ha, hb = a["normal"][:, 3] > 0.5, b["normal"][:, 3] > 0.5
    assert (ha != hb).sum() <= 3
    both = ha & hb
    rel = np.abs(a["depth64"][both] - b["depth64"][both]) / b["depth64"][both]
    assert np.percentile(rel, 99) < 1e-5


def test_edge_cases():
    # zero steps: march_to's loop never runs -> a miss
    v = _view("mandelbrot", 4, -2.5, [8.0, 12.0], max_steps=0)
    o = pyoracle.render(v, "mandelbrot", 64)
    assert (o["normal"][:, 3] == 0).all() and (o["steps"] == 0).all()
    # a tile of a frame gives the same rays as the same pixels of the whole frame
    full = _view("amazingbox_box", 40, -4.0, [-1.5, 0.5, 1.0, 1.0, 10, 0, 0, 0, 1, 0, 0, 0])
    tile = _view("amazingbox_box", 40, -4.0, [-1.5, 0.5, 1.0, 1.0, 10, 0, 0, 0, 1, 0, 0, 0],
                 tile_x=10, tile_y=5, tile_w=7, tile_h=3)
    of = pyoracle.render(full, "amazingbox_box", 64)
    ot = pyoracle.render(tile, "amazingbox_box", 64)
    idx = [(5 + y) * 40 + 10 + x for y in range(3) for x in range(7)]
    np.testing.assert_array_equal(of["depth64"][idx], ot["depth64"])
    # jittered samples are deterministic per seed
    j1 = pyoracle.render(_view("mandelbrot", 8, -2.5, [8.0, 6.0], spp=4, seed=9), "mandelbrot", 64)
    j2 = pyoracle.render(_view("mandelbrot", 8, -2.5, [8.0, 6.0], spp=4, seed=9), "mandelbrot", 64)
    np.testing.assert_array_equal(j1["depth64"], j2["depth64"])


def test_unknown_formula_raises():
    with pytest.raises(ValueError):
        pyoracle.de("no_such_formula", [0.0], np.zeros((1, 3)))


MARCH_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "march_reference_fp64.json")


def test_oracle_march_matches_the_reference_march():
    """The hand-written march (march_to, bisection, verify and high-quality modes) and
    tetrahedral normal against the reference's own march code run in FP64
    (tests/golden/march_reference_fp64.json, written by oracle/_ref)."""
    with open(MARCH_GOLDEN) as fh:
        cases = json.load(fh)["cases"]
    assert len(cases) == 18
    for c in cases:
        v = abi.make_view(0, 16, 16, tuple(c["camera"]), fov_y_deg=60.0, params=c["params"], max_steps=256,
                          **c["mode"])
        o = pyoracle.render(v, c["formula"], 64)
        hit = np.array(c["hit"]) == 1
        what = f"{c['formula']} {c['mode']}"
        np.testing.assert_array_equal(o["normal"][:, 3] > 0.5, hit, err_msg=what)
        np.testing.assert_array_equal(o["steps"], c["steps"], err_msg=what)
        np.testing.assert_array_equal(o["evals"], np.array(c["evals"]) + 4 * hit, err_msg=what)
        t = np.array(c["t"])
        rel = np.abs(o["depth64"][hit] - t[hit]) / t[hit]
        assert rel.max(initial=0.0) <= 1e-13, what
        np.testing.assert_allclose(o["normal"][hit, :3], np.array(c["normal"])[hit], atol=1e-6, err_msg=what)
        assert hit.sum() > 0 or c["formula"] == "pseudokleinian_kleinian"


TRAP_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "trap_reference_fp64.json")


def trap_desc(t):
    """nd_trap_desc from a fixture's trap record (center xyz, shape, box xyz, mode, radius, tube)."""
    d = abi.nd_trap_desc()
    d.center[:] = t[0:3]
    d.shape = int(t[3])
    d.box[:] = t[4:7]
    d.mode = int(t[7])
    d.radius, d.tube, d.span = t[8], t[9], 1.5
    return d


def test_oracle_trap_matches_the_reference_wrapper():
    """DE and orbit trap of the oracle's formula wrapper against the reference's
    generated wrapper with its trap functions, FP64 (tests/golden/trap_reference_fp64.json)."""
    with open(TRAP_GOLDEN) as fh:
        cases = json.load(fh)["cases"]
    assert len(cases) == 6 * 9
    for c in cases:
        de, tr, _ = pyoracle.de(c["formula"], c["params"], np.array(c["points"]), 64, trap=trap_desc(c["trap"]))
        what = f"{c['formula']} trap {c['trap'][3]:.0f}/{c['trap'][7]:.0f}"
        np.testing.assert_allclose(de, c["de"], rtol=1e-13, atol=1e-15, err_msg=what)
        np.testing.assert_allclose(tr, c["trap_value"], rtol=1e-13, atol=1e-15, err_msg=what)


SHADE_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "shade_reference_fp64.json")


def test_oracle_shade_and_shadow_match_the_reference():
    """The Lambert level with the camera key light and the shadow ray's visibility
    against the reference's simple_geometry and visibility_march run in FP64
    (tests/golden/shade_reference_fp64.json)."""
    with open(SHADE_GOLDEN) as fh:
        cases = json.load(fh)["cases"]
    for c in cases:
        kw = dict(shadow=1, light_dir=(0.4, 0.8, -0.45)) if c["shadow"] else {}
        v = abi.make_view(0, 16, 16, tuple(c["camera"]), fov_y_deg=90.0, params=c["params"], max_steps=256, **kw)
        o = pyoracle.render(v, c["formula"], 64)
        hit = np.array(c["hit"]) == 1
        np.testing.assert_array_equal(o["normal"][:, 3] > 0.5, hit)
        if c["shadow"]:
            dv = np.abs(o["shadow"][hit] - np.array(c["visibility"])[hit])
            # the pseudo-Kleinian's lattice DE jumps, so a shadow ray started a few
            # ulps apart (the normal is normalised with a different rounding) can take
            # other steps and even meet the surface: there most rays agree exactly
            if c["formula"] == "pseudokleinian_kleinian":
                assert (dv <= 1e-5).mean() >= 0.8, (dv <= 1e-5).mean()
            else:
                assert dv.max() <= 1e-5, (c["formula"], dv.max())
            assert (np.array(c["visibility"])[hit] < 0.99).any()
        else:
            np.testing.assert_allclose(o["shade"][hit], np.array(c["shade"])[hit], atol=1e-6)
