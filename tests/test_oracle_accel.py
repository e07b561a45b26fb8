"""The CPU oracle's empty-space accelerator (cascade placement src/gpu/accel.zig:32-56,
cs_build_accel template.wgsl:5412-5431, accel_skip :428-447 and its use in march_to
:1890-1900 and visibility_march :2297-2303) against closed forms."""

import numpy as np

from numericdream_b200 import abi
from oracle import pyoracle


def _view(size=33, cam=(0.0, 0.0, -3.0), **kw):
    kw.setdefault("eps_coef", 1e-5)
    kw.setdefault("eps_floor", 0.0)
    kw.setdefault("max_steps", 512)
    return abi.make_view(0, size, size, cam, fov_y_deg=60.0, **kw)


def _place(cam, max_dist, levels, res):
    """placeCascades restated in numpy f32."""
    f = np.float32
    res_f = f(res)
    coarsest = max(f(f(2.0) * f(max_dist)) / res_f, f(1e-6))
    out = np.zeros((8, 4), np.float32)
    for l in range(levels):
        cell = f(coarsest / f(1 << (levels - 1 - l)))
        half = f(f(f(0.5) * res_f) * cell)
        for a in range(3):
            out[l, a] = f(np.floor(f(f(cam[a]) - half) / cell) * cell)
        out[l, 3] = cell
    return out


def test_grid_of_a_sphere_is_its_exact_skip():
    # sphere primitive of radius 1: DE(c) = |c| - 1, so every voxel holds
    # max(|c| - 1 - sqrt(3)/2 cell, 0) * safety
    v = _view(cam=(0.3, -0.2, -3.1), params=[1.0], accel_res=16, accel_levels=3, accel_safety=0.92, max_dist=6.0)
    grid, prm = pyoracle.accel_grid(v, "sphere_primitive", 64)
    assert grid.shape == (3, 16, 16, 16)
    np.testing.assert_array_equal(prm, _place((0.3, -0.2, -3.1), 6.0, 3, 16))
    # every cascade holds the camera, cells halve from the coarsest (2 max_dist / res)
    assert prm[2, 3] == np.float32(0.75) and prm[1, 3] == np.float32(0.375) and prm[0, 3] == np.float32(0.1875)
    idx = np.arange(16, dtype=np.float32) + np.float32(0.5)
    for l in range(3):
        cell = prm[l, 3]
        cx = (prm[l, 0] + idx * cell).astype(np.float32)
        cy = (prm[l, 1] + idx * cell).astype(np.float32)
        cz = (prm[l, 2] + idx * cell).astype(np.float32)
        z, y, x = np.meshgrid(cz, cy, cx, indexing="ij")
        d = np.sqrt(x.astype(np.float64) ** 2 + y.astype(np.float64) ** 2 + z.astype(np.float64) ** 2) - 1.0
        want = np.maximum(d.astype(np.float32) - np.float32(0.8660254) * cell, 0) * np.float32(0.92)
        np.testing.assert_allclose(grid[l], want, rtol=1e-6, atol=1e-6)


def test_resolution_and_levels_are_clamped():
    v = _view(params=[1.0], accel_res=7, accel_levels=20, accel_safety=1.0)
    grid, prm = pyoracle.accel_grid(v, "sphere_primitive", 64)
    assert grid.shape == (8, 16, 16, 16)
    v.accel_res, v.accel_levels = 167, 0
    grid, prm = pyoracle.accel_grid(v, "sphere_primitive", 64)
    assert grid.shape == (1, 160, 160, 160)
    v.accel_res = 66
    assert pyoracle.accel_grid(v, "sphere_primitive", 64)[0].shape == (1, 64, 64, 64)


def test_accelerated_march_of_exact_sdfs_keeps_every_hit_and_saves_evaluations():
    # sphere tracing an exact SDF with safe skips: the same rays hit, each hit lies
    # within eps(t) of the surface, and the empty space costs fewer evaluations
    for name, prm in (("sphere_primitive", [1.0]), ("cube_primitive", [0.7])):
        v = _view(49, cam=(0.4, 0.3, -4.0), params=prm)
        a = pyoracle.render(v, name, 64)
        v.accel_res, v.accel_levels, v.accel_safety = 32, 4, 0.92
        b = pyoracle.render(v, name, 64)
        ha, hb = a["normal"][:, 3] > 0.5, b["normal"][:, 3] > 0.5
        np.testing.assert_array_equal(ha, hb)
        rel = np.abs(a["depth64"][ha] - b["depth64"][ha]) / a["depth64"][ha]
        assert rel.max() <= 3e-5, name
        assert b["evals"].sum() < 0.8 * a["evals"].sum(), name
        assert (b["evals"] <= a["evals"]).mean() > 0.95


def test_sphere_hit_distance_with_the_accelerator_known_answer():
    R, cz = 1.25, -3.0
    v = _view(65, cam=(0.0, 0.0, cz), params=[R], accel_res=64, accel_levels=6)
    o = pyoracle.render(v, "sphere_primitive", 64)
    c = 32 * 65 + 32
    t = abs(cz) - R
    assert o["normal"][c, 3] == 1.0
    assert t - 1e-5 * t <= o["depth64"][c] <= t + 1e-12


def test_shadow_rays_take_the_accelerator_jumps():
    # a cube lit from the side: shadow visibility with and without the accelerator
    # agrees where it is 0 or 1 and costs fewer evaluations
    v = _view(33, cam=(0.6, 0.8, -3.0), params=[0.6], shadow=1, light_dir=(0.4, 0.9, -0.3))
    a = pyoracle.render(v, "cube_primitive", 64)
    v.accel_res, v.accel_levels = 32, 4
    b = pyoracle.render(v, "cube_primitive", 64)
    hit = a["normal"][:, 3] > 0.5
    np.testing.assert_array_equal(hit, b["normal"][:, 3] > 0.5)
    lit = hit & (a["shadow"] == 1.0)
    assert lit.sum() > 50
    assert (b["shadow"][lit] > 0.99).mean() > 0.95
    assert b["evals"][hit].sum() < a["evals"][hit].sum()


def test_scene_grid_uses_the_scene_de():
    names = {0: "sphere_primitive"}.get
    v = _view(33, cam=(0.0, 0.0, -3.0), accel_res=32, accel_levels=4)
    a = abi.make_instance(0, params=[1.0], offset=(0.5, 0.0, 0.0), scale=(0.5, 0.5, 0.5))
    b = abi.make_instance(0, params=[1.0], offset=(-0.5, 0.0, 0.0), scale=(0.5, 0.5, 0.5))
    scene = abi.make_scene([a, b])
    on = pyoracle.render_scene(v, scene, names, 64)
    v.accel_res = 0
    off = pyoracle.render_scene(v, scene, names, 64)
    np.testing.assert_array_equal(on["normal"][:, 3], off["normal"][:, 3])
    assert on["evals"].sum() < off["evals"].sum()
    # the centre ray runs down the gap between the spheres to where they touch, at
    # t = 3: the DE there is ~ z^2, under eps(t) = 3e-5 from |z| < 0.0055 on
    c = 16 * 33 + 16
    assert on["normal"][c, 3] == 1.0 and 3.0 - 0.006 <= on["depth64"][c] <= 3.0
    assert abs(on["depth64"][c] - off["depth64"][c]) <= 1e-4
