"""The CPU oracle's multi-instance scene path (scene_de, template.wgsl:1756-1779):
equivalence with the single-instance march, and closed-form answers for placed,
scaled, rotated and carved primitives."""

import math

import numpy as np

from numericdream_b200 import abi
from oracle import pyoracle

# formula ids of these tests -> oracle formula names (the oracle takes names)
NAMES = {0: "sphere_primitive", 1: "cube_primitive", 2: "mandelbrot", 3: "amazingbox_box"}


def _view(size=33, cam_z=-3.0, **kw):
    kw.setdefault("eps_coef", 1e-5)
    kw.setdefault("eps_floor", 0.0)
    kw.setdefault("max_steps", 512)
    return abi.make_view(0, size, size, (0.0, 0.0, cam_z), fov_y_deg=60.0, **kw)


def _hit(o, i):
    return o["normal"][i, 3] > 0.5


def test_identity_instance_equals_the_plain_march():
    prm = [8.0, 10.0]
    v = _view(40, -2.6, params=prm, eps_coef=5e-4, eps_floor=5e-5)
    inst = abi.make_instance(2, params=prm)
    inst.trap = v.trap
    a = pyoracle.render(v, "mandelbrot", 64)
    b = pyoracle.render_scene(v, abi.make_scene([inst]), NAMES.get, 64)
    for k in ("depth64", "steps", "evals", "iters", "normal", "trap", "shade"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_hidden_instance_contributes_nothing():
    v = _view(24, -3.0)
    a = abi.make_instance(0, params=[1.0])
    b = abi.make_instance(1, params=[0.5], offset=(0.0, 0.0, -1.5), hidden=True)
    one = pyoracle.render_scene(v, abi.make_scene([a]), NAMES.get, 64)
    two = pyoracle.render_scene(v, abi.make_scene([a, b]), NAMES.get, 64)
    np.testing.assert_array_equal(one["depth64"], two["depth64"])


def test_offset_and_scaled_sphere_known_answer():
    # unit sphere scaled by 1.5 and moved to (0.3, 0, 0): the centre ray from
    # (0, 0, -3) along +z meets it at z = -sqrt(1.5^2 - 0.3^2)
    v = _view(33, -3.0)
    inst = abi.make_instance(0, params=[1.0], offset=(0.3, 0.0, 0.0), scale=(1.5, 1.5, 1.5))
    o = pyoracle.render_scene(v, abi.make_scene([inst]), NAMES.get, 64)
    c = 16 * 33 + 16
    t = 3.0 - math.sqrt(1.5 ** 2 - 0.3 ** 2)
    assert _hit(o, c)
    assert t - 2e-5 * t <= o["depth64"][c] <= t + 1e-12
    # the normal at that point points from the sphere's centre to it
    p = np.array([0.0, 0.0, -3.0 + o["depth64"][c]])
    n = (p - np.array([0.3, 0.0, 0.0])) / 1.5
    np.testing.assert_allclose(o["normal"][c, :3], n, atol=1e-4)


def test_rotated_cube_known_answer():
    # a cube of half size 0.6 turned 45 degrees about y shows an edge to the camera
    # at distance 0.6 * sqrt(2) from its centre
    v = _view(33, -3.0)
    inst = abi.make_instance(1, params=[0.6], rotation_deg=(0.0, 45.0, 0.0))
    o = pyoracle.render_scene(v, abi.make_scene([inst]), NAMES.get, 64)
    c = 16 * 33 + 16
    t = 3.0 - 0.6 * math.sqrt(2.0)
    assert _hit(o, c)
    assert abs(o["depth64"][c] - t) <= 2e-5 * t + 1e-9


def test_rotation_frame_is_orthonormal_and_composes_x_then_y_then_z():
    f = np.array(abi.rotation_frame(30.0, -50.0, 110.0)).reshape(3, 3).T  # columns -> matrix
    np.testing.assert_allclose(f @ f.T, np.eye(3), atol=1e-12)
    assert abs(np.linalg.det(f) - 1.0) < 1e-12

    def rot(axis, deg):
        a = math.radians(deg)
        c, s = math.cos(a), math.sin(a)
        return {"x": np.array([[1, 0, 0], [0, c, -s], [0, s, c]]),
                "y": np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]]),
                "z": np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])}[axis]

    np.testing.assert_allclose(f, rot("z", 110.0) @ rot("y", -50.0) @ rot("x", 30.0), atol=1e-12)


def test_union_smooth_union_and_carve():
    v = _view(33, -3.0)
    c = 16 * 33 + 16
    a = abi.make_instance(0, params=[0.5], offset=(0.0, 0.45, 0.0))
    b = abi.make_instance(0, params=[0.5], offset=(0.0, -0.45, 0.0))
    union = pyoracle.render_scene(v, abi.make_scene([a, b]), NAMES.get, 64)
    # the centre ray passes between the spheres' surfaces at (0, 0, z): the sphere
    # centred 0.45 away with radius 0.5 reaches z = -sqrt(0.25 - 0.2025)
    # (oblique incidence: the march stops up to eps(t) / cos short, cos = chord / r)
    t = 3.0 - math.sqrt(0.25 - 0.45 ** 2)
    cos_inc = math.sqrt(0.25 - 0.45 ** 2) / 0.5
    assert _hit(union, c) and t - 1.1e-5 * t / cos_inc <= union["depth64"][c] <= t + 1e-12
    b.combine_mode, b.blend_k = abi.ND_COMBINE_SMOOTH_MIN, 0.3
    smooth = pyoracle.render_scene(v, abi.make_scene([a, b]), NAMES.get, 64)
    assert _hit(smooth, c) and smooth["depth64"][c] < union["depth64"][c] - 0.01  # the blend fills the gap
    hs, hu = smooth["normal"][:, 3] > 0.5, union["normal"][:, 3] > 0.5
    assert (hs | ~hu).all() and hs.sum() > hu.sum()  # smooth min <= min: every union hit stays a hit
    # a carve sphere of radius 0.4 at the front of the blend pushes the centre hit back
    carved = pyoracle.render_scene(v, abi.make_scene([a, b], carves=[(0.0, 0.0, -0.3, 0.4)]), NAMES.get, 64)
    assert carved["depth64"][c] > smooth["depth64"][c] + 0.1 or not _hit(carved, c)


def test_combine_modes_and_carves_against_numpy():
    # the DE of two spheres and a carve at random points, mode by mode, against
    # numpy restatements of the smooth operators (template.wgsl:1648-1753)
    k = 0.25

    def mix(a, b, h):
        return a * (1 - h) + b * h

    def smin(a, b):
        h = np.clip(0.5 + 0.5 * (b - a) / k, 0, 1)
        return mix(b, a, h) - k * h * (1 - h)

    def smax(a, b):
        h = np.clip(0.5 - 0.5 * (b - a) / k, 0, 1)
        return mix(b, a, h) + k * h * (1 - h)

    def ssub(cut, base, kk):
        h = np.clip(0.5 - 0.5 * (base + cut) / kk, 0, 1)
        return mix(base, -cut, h) + kk * h * (1 - h)

    def slin(a, b):
        return np.minimum(b - np.maximum(k - a, 0), a - np.maximum(k - b, 0))

    def snlin(a, b):
        ra, rb = np.maximum(k - a, 0), np.maximum(k - b, 0)
        return np.minimum(b - ra * (k - rb) / k, a - rb * (k - ra) / k)

    def smix(a, b):
        h = np.clip(0.5 + 0.5 * (b - a) / k, 0, 1)
        return mix(b, a, h)

    ops = {abi.ND_COMBINE_UNION: np.minimum, abi.ND_COMBINE_SMOOTH_MIN: smin, abi.ND_COMBINE_SMOOTH_MAX: smax,
           abi.ND_COMBINE_SMOOTH_INV_MAX: lambda d, di: ssub(di, d, k), abi.ND_COMBINE_SMOOTH_MIN_LIN: slin,
           abi.ND_COMBINE_SMOOTH_MIN_NLIN: snlin, abi.ND_COMBINE_SMOOTH_MIX: smix}
    rng = np.random.default_rng(5)
    pts = rng.uniform(-1.5, 1.5, (4000, 3))
    f32 = lambda x: np.float32(x).astype(np.float64)  # the scene is described in f32
    ca, ra = f32([0.0, 0.3, 0.0]), float(f32(0.5))
    cb, rb = f32([0.1, -0.2, 0.2]), float(f32(0.6))
    da = np.linalg.norm(pts - ca, axis=1) - ra
    db = np.linalg.norm(pts - cb, axis=1) - rb
    carve = tuple(float(x) for x in f32([0.2, 0.0, -0.4, 0.35]))
    dc = np.linalg.norm(pts - np.array(carve[:3]), axis=1) - carve[3]
    for mode, op in ops.items():
        a = abi.make_instance(0, params=[1.0], offset=tuple(ca), scale=(ra,) * 3)
        b = abi.make_instance(0, params=[1.0], offset=tuple(cb), scale=(rb,) * 3, combine_mode=mode, blend_k=k)
        got, _, _ = pyoracle.scene_de(abi.make_scene([a, b]), NAMES.get, pts)
        np.testing.assert_allclose(got, op(da, db), rtol=1e-12, atol=1e-12, err_msg=str(mode))
        got, _, _ = pyoracle.scene_de(abi.make_scene([a, b], carves=[carve]), NAMES.get, pts)
        np.testing.assert_allclose(got, ssub(dc, op(da, db), 0.2 * carve[3]), rtol=1e-12, atol=1e-12)
    # an instance with every instance hidden is the empty scene: 2 max_dist + 1
    h = abi.make_instance(0, params=[1.0], hidden=True)
    got, _, _ = pyoracle.scene_de(abi.make_scene([h]), NAMES.get, pts[:5], max_dist=10.0)
    assert (got == 21.0).all()
    # the trap follows the nearest visible instance
    ta = abi.make_instance(0, params=[1.0], offset=(-2.0, 0.0, 0.0), trap={"center": [5.0, 0.0, 0.0]})
    tb = abi.make_instance(0, params=[1.0], offset=(2.0, 0.0, 0.0), trap={"center": [0.0, 7.0, 0.0]})
    _, tr, _ = pyoracle.scene_de(abi.make_scene([ta, tb]), NAMES.get, [[-1.5, 0, 0], [1.5, 0, 0]])
    # the primitive's one step rescales z to the unit sphere frame: |z - c| at the local point
    assert abs(tr[0] - np.linalg.norm(np.array([0.5, 0, 0]) - [5.0, 0, 0])) < 1e-12
    assert abs(tr[1] - np.linalg.norm(np.array([-0.5, 0, 0]) - [0.0, 7.0, 0])) < 1e-12


def test_hybrid_mixin_iteration_schedule():
    # base Mandelbox for 2 iterations, then a Mandelbulb mixin for 1, cycled 10
    # times; as a DE value check against an explicit evaluation of the schedule with
    # the oracle's single-formula steps: the hybrid with mixin iterations 0 and
    # total = base iterations equals the base formula with that iteration count
    box = [-1.5, 0.5, 1.0, 1.0, 7, 0, 0, 0, 1, 0, 0, 0]
    v = _view(24, -4.0, params=box, eps_coef=5e-4, eps_floor=5e-5)
    plain = abi.make_instance(3, params=box)
    plain.trap = v.trap
    hyb = abi.make_instance(3, params=box, mixins=[(2, 0, [8.0, 4.0])], hybrid_base_iters=7, hybrid_total_iters=7)
    hyb.trap = v.trap
    a = pyoracle.render_scene(v, abi.make_scene([plain]), NAMES.get, 64)
    b = pyoracle.render_scene(v, abi.make_scene([hyb]), NAMES.get, 64)
    for key in ("depth64", "steps", "evals", "trap", "iters"):
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)
    # a real mixin changes the surface
    mixed = abi.make_instance(3, params=box, mixins=[(2, 1, [8.0, 4.0])], hybrid_base_iters=2, hybrid_total_iters=9)
    m = pyoracle.render_scene(v, abi.make_scene([mixed]), NAMES.get, 64)
    assert (m["depth64"] != a["depth64"]).any()
