"""Scene files (.dream JSON, src/app/scene_file.zig) through nd_scene_file_load: the
descriptors it fills (camera basis, bench-export march settings, instances with
formulas by file stem, @param values by name over the defaults, placement, combine
modes, mixins, orbit traps) and its refusals.  tests/golden/two_fractals.dream is a
scene written for these tests in the reference's version-12 format."""

import json
import math
import os

import numpy as np
import pytest

from numericdream_b200 import abi, runtime

HERE = os.path.dirname(os.path.abspath(__file__))
SCENE = os.path.join(HERE, "golden", "two_fractals.dream")


def _minimal(**over):
    d = {"version": 12,
         "camera": {"position": {"x": 0, "y": 0, "z": 3}, "forward": {"x": 0, "y": 0, "z": -1},
                    "up": {"x": 0, "y": 1, "z": 0}},
         "export_width": 64, "export_height": 48,
         "instances": [{"formula": {"path": "", "params": []}}]}
    d.update(over)
    return json.dumps(d)


def test_scene_file_fields(ndlib):
    v, s = runtime.load_scene_file(SCENE)
    assert s is not None and s.instance_count == 2
    # camera: position / forward / up as saved (f32), right = normalize(forward x up)
    f = np.array([-0.0688, -0.1376, -0.9881], np.float32)
    u = np.array([-0.0096, 0.9905, -0.1373], np.float32)
    r = np.cross(f.astype(np.float64), u.astype(np.float64))
    np.testing.assert_allclose(v.right[:], r / np.linalg.norm(r), atol=1e-6)
    np.testing.assert_allclose(v.cam_pos[:], [0.25, 0.5, 3.6], atol=1e-6)
    assert (v.width, v.height, v.tile_w, v.tile_h, v.spp) == (320, 180, 320, 180, 1)
    # the bench export's settings: render_settings and its precision, high quality
    assert (v.max_steps, v.max_dist, v.refine_budget, v.high_quality, v.march_verify) == (200, 16.0, 12, 1, 0)
    assert abs(v.eps_coef - 4e-4) < 1e-9 and abs(v.eps_floor - 2e-5) < 1e-10 and abs(v.hq_footprint_px - 1.5) < 1e-7
    # instance 0: built-in Mandelbulb, Power by name over the default Iterations
    a, b = s.instances[0], s.instances[1]
    assert runtime.formula_name(a.formula) == "mandelbrot" and v.formula == a.formula
    defaults = [p.default_value for p in runtime.formula_params(a.formula)]
    assert list(a.params[:2]) == [7.5, defaults[1]]
    assert list(v.params[:2]) == list(a.params[:2])
    np.testing.assert_allclose(a.offset[:], [-0.8, 0, 0], atol=1e-7)
    np.testing.assert_allclose(a.scale[:], [0.7] * 3, atol=1e-7)
    np.testing.assert_allclose(a.frame[:], abi.rotation_frame(15, -25, 5), atol=1e-6)
    assert abs(a.step_safety - 0.9) < 1e-7 and a.combine_mode == abi.ND_COMBINE_UNION
    assert (a.hybrid_base_iters, a.hybrid_total_iters, a.mixin_count, a.hidden) == (1, 8, 0, 0)
    t = a.trap
    assert (t.shape, t.mode, t.repeat) == (abi.ND_TRAP_SPHERE, abi.ND_TRAP_AVERAGE, 2)
    np.testing.assert_allclose(t.center[:], [0.1, 0.2, 0.3], atol=1e-7)
    assert (round(t.radius, 6), round(t.tube, 6), t.span, t.offset) == (0.8, 0.1, 2.0, 0.25)
    # instance 1: path stem, scale x scale_uniform, smooth min, a Menger mixin
    assert runtime.formula_name(b.formula) == "amazingbox_box"
    box_defaults = [p.default_value for p in runtime.formula_params(b.formula)]
    assert list(b.params[:12]) == [np.float32(x) for x in box_defaults[:4] + [9.0] + box_defaults[5:12]]
    np.testing.assert_allclose(b.scale[:], [0.4] * 3, atol=1e-7)
    assert b.combine_mode == abi.ND_COMBINE_SMOOTH_MIN and abs(b.blend_k - 0.2) < 1e-7
    assert b.mixin_count == 1 and b.mixins[0].iterations == 1
    assert runtime.formula_name(b.mixins[0].formula) == "menger3_ifs"
    menger = [p.default_value for p in runtime.formula_params(b.mixins[0].formula)]
    assert list(b.mixins[0].params[:len(menger)]) == [np.float32(x) for x in menger]
    # the default trap (OrbitTrapState): point, min, clamp, radius 1, span 1.5
    assert (b.trap.shape, b.trap.mode, b.trap.repeat, b.trap.radius, b.trap.span) == (0, 0, 0, 1.0, 1.5)


def test_identity_single_instance_needs_no_scene(ndlib):
    v, s = runtime.load_scene_file(_minimal(), 40, 30)
    assert s is None and (v.width, v.height) == (40, 30)
    assert runtime.formula_name(v.formula) == "mandelbrot"
    assert list(v.params[:2]) == [p.default_value for p in runtime.formula_params(v.formula)][:2]
    # defaults of RenderSettingsState / MarchPrecision when the file has none
    assert (v.max_steps, v.max_dist, v.refine_budget, v.high_quality) == (256, 24.0, 20, 1)
    assert abs(v.eps_coef - 5e-4) < 1e-9
    # a 90 degree vertical field of view: right and up are unit vectors
    assert abs(math.sqrt(sum(x * x for x in v.right)) - 1) < 1e-6
    # hidden, moved or hybrid instances need the scene path
    d = json.loads(_minimal())
    d["instances"][0]["visible"] = False
    assert runtime.load_scene_file(json.dumps(d))[1] is not None
    d = json.loads(_minimal())
    d["instances"][0]["rotation"] = {"x": 0, "y": 10, "z": 0}
    assert runtime.load_scene_file(json.dumps(d))[1] is not None


def test_scene_file_refusals(ndlib):
    with pytest.raises(runtime.NDError) as e:
        runtime.load_scene_file('{"version": 12, "camera": ')
    assert e.value.status == abi.ND_ERR_INVALID and "JSON" in str(e.value)
    with pytest.raises(runtime.NDError) as e:
        runtime.load_scene_file(_minimal(version=13))
    assert e.value.status == abi.ND_ERR_UNSUPPORTED
    d = json.loads(_minimal())
    d["instances"][0]["formula"]["path"] = "formulas/no_such_formula.wgsl"
    with pytest.raises(runtime.NDError) as e:
        runtime.load_scene_file(json.dumps(d))
    assert e.value.status == abi.ND_ERR_NOT_FOUND and "no_such_formula" in str(e.value)
    d = json.loads(_minimal())
    del d["camera"]["up"]
    with pytest.raises(runtime.NDError) as e:
        runtime.load_scene_file(json.dumps(d))
    assert "camera.up" in str(e.value)
    d = json.loads(_minimal())
    d["instances"][0]["combine_mode"] = "blend"
    with pytest.raises(runtime.NDError) as e:
        runtime.load_scene_file(json.dumps(d))
    assert "combine_mode" in str(e.value)
    d = json.loads(_minimal())
    del d["export_width"]
    with pytest.raises(runtime.NDError):
        runtime.load_scene_file(json.dumps(d))
    # JSON escapes and unicode in strings parse
    d = json.loads(_minimal())
    d["note"] = "café \"quoted\" \\ 😀"
    runtime.load_scene_file(json.dumps(d))


def test_scene_file_lite(ndlib):
    lite = runtime.load_scene_file_lite(SCENE)
    assert (lite.color_count, lite.light_count, lite.ambient_occlusion, lite.specular) == (2, 2, 1, 1)
    # stops as saved (the shading call sorts them by position)
    assert lite.colors[0].position == 1.0 and lite.colors[1].position == 0.0
    np.testing.assert_allclose(lite.colors[1].color[:], [0.1, 0.2, 0.5], atol=1e-7)
    assert abs(lite.colors[0].glossiness - 0.7) < 1e-7 and abs(lite.colors[0].ior - 1.6) < 1e-7
    # the global light's direction, the point light's position; the ray light and the
    # hidden light are left out
    a, b = lite.lights[0], lite.lights[1]
    assert a.type == abi.ND_LIGHT_GLOBAL and b.type == abi.ND_LIGHT_POINT
    np.testing.assert_allclose(a.position_or_direction[:], [-0.4, 0.8, 0.3], atol=1e-7)
    np.testing.assert_allclose(b.position_or_direction[:], [1.5, 2.0, 2.5], atol=1e-7)
    assert (a.brightness, b.brightness) == (1.5, 4.0)
    np.testing.assert_allclose(lite.background[:], [0.10, 0.11, 0.13], atol=1e-7)
    # a scene without stops or lights: the default material, no lights
    bare = runtime.load_scene_file_lite(_minimal())
    assert (bare.color_count, bare.light_count) == (0, 0)


class _GuardedText:
    """Bytes placed so that they end where an inaccessible page begins: a parser that
    reads one byte past the length it was given faults at once."""

    def __init__(self, data: bytes):
        import ctypes as C

        self.C = C
        libc = C.CDLL(None, use_errno=True)
        libc.mmap.restype = C.c_void_p
        libc.mmap.argtypes = [C.c_void_p, C.c_size_t, C.c_int, C.c_int, C.c_int, C.c_long]
        libc.mprotect.argtypes = [C.c_void_p, C.c_size_t, C.c_int]
        libc.munmap.argtypes = [C.c_void_p, C.c_size_t]
        self.libc = libc
        page = 4096
        self.size = ((len(data) + page - 1) // page + 1) * page
        base = libc.mmap(None, self.size, 3, 0x22, -1, 0)  # PROT_READ|WRITE, MAP_PRIVATE|ANONYMOUS
        assert base not in (None, C.c_void_p(-1).value)
        assert libc.mprotect(base + self.size - page, page, 0) == 0  # PROT_NONE
        self.base = base
        self.addr = base + self.size - page - len(data)
        C.memmove(self.addr, data, len(data))
        self.n = len(data)

    def ptr(self):
        return self.C.cast(self.addr, self.C.c_char_p)

    def close(self):
        self.libc.munmap(self.base, self.size)


def test_mutated_scene_files_never_crash(ndlib):
    """Seeded byte mutations and truncations of the fixture: the loader returns a status
    (or a scene) for every one; the first 400 sit against an inaccessible page, so a
    read past the given length would fault the test process."""
    import ctypes as C
    import random

    src = open(SCENE, "rb").read()
    rng = random.Random(12345)
    alphabet = b'{}[]",:0123456789.-eE ntfulrasx\\'
    outcomes = {"ok": 0, "error": 0}
    for trial in range(3000):
        s = bytearray(src)
        for _ in range(rng.randint(1, 6)):
            i = rng.randrange(len(s))
            op = rng.random()
            if op < 0.3:
                del s[i:i + rng.randint(1, 20)]
            elif op < 0.6:
                s.insert(i, rng.choice(alphabet))
            elif op < 0.8:
                s[i] = rng.choice(alphabet)
            else:
                j = rng.randrange(len(s))
                s[i:i] = s[j:j + rng.randint(1, 40)]
        if rng.random() < 0.2:
            s = s[:rng.randrange(len(s))]
        if trial < 400:
            g = _GuardedText(bytes(s))
            try:
                view, scene, needs = abi.nd_view_desc(), abi.nd_scene_desc(), C.c_int32()
                err = C.create_string_buffer(256)
                st = ndlib.nd_scene_file_load(g.ptr(), g.n, 64, 48, C.byref(view), C.byref(scene),
                                              C.byref(needs), err, 256)
                lite = abi.nd_lite_desc()
                st2 = ndlib.nd_scene_file_lite(g.ptr(), g.n, 0, C.byref(lite), err, 256)
                assert st in (abi.ND_OK, abi.ND_ERR_INVALID, abi.ND_ERR_UNSUPPORTED, abi.ND_ERR_NOT_FOUND)
                assert st2 in (abi.ND_OK, abi.ND_ERR_INVALID, abi.ND_ERR_UNSUPPORTED, abi.ND_ERR_NOT_FOUND)
            finally:
                g.close()
        for load in (lambda: runtime.load_scene_file(bytes(s), 64, 48),
                     lambda: runtime.load_scene_file_lite(bytes(s), rng.randint(-1, 4))):
            try:
                load()
                outcomes["ok"] += 1
            except runtime.NDError as e:
                assert e.status in (abi.ND_ERR_INVALID, abi.ND_ERR_UNSUPPORTED, abi.ND_ERR_NOT_FOUND)
                outcomes["error"] += 1
    assert outcomes["ok"] > 0 and outcomes["error"] > 0
