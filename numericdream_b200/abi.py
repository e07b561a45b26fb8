"""ctypes mirror of include/nd_march.h and helpers to fill its descriptors.

The structures here must match the C header byte for byte; ``check_layout`` is
called by the tests and compares sizes and offsets against the values the C
library reports for itself.
"""

from __future__ import annotations

import ctypes as C
import math

ND_MAX_PARAMS = 16
ND_PARAM_NAME_LEN = 24

ND_OK, ND_ERR_INVALID, ND_ERR_COMPILE, ND_ERR_OOM, ND_ERR_TIMEOUT, ND_ERR_CUDA, ND_ERR_UNSUPPORTED, ND_ERR_NOT_FOUND = range(8)
STATUS_NAMES = ["ND_OK", "ND_ERR_INVALID", "ND_ERR_COMPILE", "ND_ERR_OOM", "ND_ERR_TIMEOUT", "ND_ERR_CUDA",
                "ND_ERR_UNSUPPORTED", "ND_ERR_NOT_FOUND"]

ND_TRAP_POINT, ND_TRAP_SPHERE, ND_TRAP_BOX, ND_TRAP_CROSS, ND_TRAP_TORUS = range(5)
ND_TRAP_MIN, ND_TRAP_MAX, ND_TRAP_AVERAGE, ND_TRAP_LAST, ND_TRAP_ITERATION = range(5)
ND_NORMAL_TETRA, ND_NORMAL_CENTRAL = 0, 1
ND_KERNEL_AUTO, ND_KERNEL_PLAIN, ND_KERNEL_PERSISTENT = 0, 1, 2
ND_VIEW_DIR64 = 1
ND_VIEW_EXACT_HIT = 2


class nd_param_info(C.Structure):
    _fields_ = [("name", C.c_char * ND_PARAM_NAME_LEN), ("min_value", C.c_float), ("max_value", C.c_float),
                ("default_value", C.c_float), ("integral", C.c_int32)]


class nd_trap_desc(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("shape", C.c_int32), ("box", C.c_float * 3), ("mode", C.c_int32),
                ("radius", C.c_float), ("tube", C.c_float), ("span", C.c_float), ("offset", C.c_float),
                ("repeat", C.c_int32), ("reserved", C.c_int32)]


class nd_view_desc(C.Structure):
    _fields_ = [
        ("cam_pos", C.c_double * 3), ("fwd", C.c_double * 3), ("right", C.c_double * 3), ("up", C.c_double * 3),
        ("width", C.c_int32), ("height", C.c_int32), ("tile_x", C.c_int32), ("tile_y", C.c_int32),
        ("tile_w", C.c_int32), ("tile_h", C.c_int32), ("formula", C.c_int32), ("spp", C.c_int32),
        ("seed", C.c_uint64), ("params", C.c_float * ND_MAX_PARAMS), ("trap", nd_trap_desc),
        ("max_steps", C.c_int32), ("max_dist", C.c_float), ("eps_coef", C.c_float), ("eps_floor", C.c_float),
        ("refine_budget", C.c_int32), ("march_verify", C.c_int32), ("high_quality", C.c_int32),
        ("hq_footprint_px", C.c_float), ("normal_mode", C.c_int32), ("normal_h_coef", C.c_float),
        ("shadow", C.c_int32), ("light_dir", C.c_float * 3), ("shadow_k", C.c_float), ("step_safety", C.c_float),
        ("flags", C.c_int32), ("accel_res", C.c_int32), ("accel_levels", C.c_int32), ("accel_safety", C.c_float),
        ("image_texels", C.c_void_p), ("image_width", C.c_int32), ("image_height", C.c_int32),
        ("image_slope", C.c_float * 4),
    ]


ND_MAX_INSTANCES, ND_MAX_MIXINS, ND_MAX_CARVES = 4, 3, 16
(ND_COMBINE_UNION, ND_COMBINE_SMOOTH_MIN, ND_COMBINE_SMOOTH_MAX, ND_COMBINE_SMOOTH_INV_MAX, ND_COMBINE_SMOOTH_MIN_LIN,
 ND_COMBINE_SMOOTH_MIN_NLIN, ND_COMBINE_SMOOTH_MIX) = range(7)


class nd_mixin_desc(C.Structure):
    _fields_ = [("formula", C.c_int32), ("iterations", C.c_int32), ("params", C.c_float * ND_MAX_PARAMS)]


class nd_instance_desc(C.Structure):
    _fields_ = [("formula", C.c_int32), ("hidden", C.c_int32), ("params", C.c_float * ND_MAX_PARAMS),
                ("offset", C.c_float * 3), ("scale", C.c_float * 3), ("frame", C.c_float * 9),
                ("step_safety", C.c_float), ("blend_k", C.c_float), ("combine_mode", C.c_int32),
                ("mixin_count", C.c_int32), ("hybrid_base_iters", C.c_int32), ("hybrid_total_iters", C.c_int32),
                ("mixins", nd_mixin_desc * ND_MAX_MIXINS), ("trap", nd_trap_desc)]


class nd_scene_desc(C.Structure):
    _fields_ = [("instance_count", C.c_int32), ("carve_count", C.c_int32),
                ("instances", nd_instance_desc * ND_MAX_INSTANCES), ("carves", (C.c_float * 4) * ND_MAX_CARVES)]


def rotation_frame(rx_deg=0.0, ry_deg=0.0, rz_deg=0.0):
    """The instance frame rot_z * rot_y * rot_x (template.wgsl:1392-1408; angles in
    degrees), as three columns."""
    def rx(a):
        c, s = math.cos(a), math.sin(a)
        return [[1, 0, 0], [0, c, s], [0, -s, c]]  # columns

    def ry(a):
        c, s = math.cos(a), math.sin(a)
        return [[c, 0, -s], [0, 1, 0], [s, 0, c]]

    def rz(a):
        c, s = math.cos(a), math.sin(a)
        return [[c, s, 0], [-s, c, 0], [0, 0, 1]]

    def mul(a, b):  # column-major 3x3: column j of a * b is a * (column j of b)
        return [[sum(a[k][i] * b[j][k] for k in range(3)) for i in range(3)] for j in range(3)]

    m = mul(rz(math.radians(rz_deg)), mul(ry(math.radians(ry_deg)), rx(math.radians(rx_deg))))
    return [m[c][r] for c in range(3) for r in range(3)]


def make_instance(formula: int, params=None, offset=(0.0, 0.0, 0.0), scale=(1.0, 1.0, 1.0), rotation_deg=(0.0, 0.0, 0.0),
                  step_safety=1.0, blend_k=0.0, combine_mode=ND_COMBINE_UNION, hidden=False, mixins=(),
                  hybrid_base_iters=0, hybrid_total_iters=0, trap=None) -> nd_instance_desc:
    """One scene instance; mixins: [(formula, iterations, params), ...]."""
    d = nd_instance_desc()
    d.formula = formula
    d.hidden = 1 if hidden else 0
    for i, p in enumerate((params or [])[:ND_MAX_PARAMS]):
        d.params[i] = p
    d.offset[:] = [float(x) for x in offset]
    d.scale[:] = [float(x) for x in scale]
    d.frame[:] = rotation_frame(*rotation_deg)
    d.step_safety, d.blend_k, d.combine_mode = step_safety, blend_k, combine_mode
    d.mixin_count = len(mixins)
    for j, (f, n, prm) in enumerate(mixins):
        d.mixins[j].formula = f
        d.mixins[j].iterations = n
        for i, p in enumerate(prm[:ND_MAX_PARAMS]):
            d.mixins[j].params[i] = p
    d.hybrid_base_iters, d.hybrid_total_iters = hybrid_base_iters, hybrid_total_iters
    d.trap.shape = ND_TRAP_POINT
    d.trap.radius = 1.0
    d.trap.box[:] = [1.0, 1.0, 1.0]
    d.trap.span = 1.5
    for k, v in (trap or {}).items():
        if k in ("center", "box"):
            getattr(d.trap, k)[:] = v
        else:
            setattr(d.trap, k, v)
    return d


def make_scene(instances, carves=()) -> nd_scene_desc:
    """A scene of 1..4 instances and up to 16 carves (x, y, z, radius)."""
    s = nd_scene_desc()
    s.instance_count = len(instances)
    for i, inst in enumerate(instances):
        s.instances[i] = inst
    s.carve_count = len(carves)
    for i, c in enumerate(carves):
        s.carves[i][:] = [float(x) for x in c]
    return s


ND_MAX_COLOR_STOPS, ND_MAX_LIGHTS = 16, 8
ND_LIGHT_POINT, ND_LIGHT_GLOBAL = 0, 1


class nd_color_stop(C.Structure):
    _fields_ = [("color", C.c_float * 3), ("position", C.c_float), ("glossiness", C.c_float), ("ior", C.c_float),
                ("reserved", C.c_float * 2)]


class nd_light(C.Structure):
    _fields_ = [("color", C.c_float * 3), ("brightness", C.c_float), ("position_or_direction", C.c_float * 3),
                ("type", C.c_int32)]


class nd_lite_desc(C.Structure):
    _fields_ = [("color_count", C.c_int32), ("light_count", C.c_int32), ("ambient_occlusion", C.c_int32),
                ("specular", C.c_int32), ("background", C.c_float * 3), ("reserved", C.c_int32),
                ("colors", nd_color_stop * ND_MAX_COLOR_STOPS), ("lights", nd_light * ND_MAX_LIGHTS)]


def make_lite(colors=(), lights=(), ambient_occlusion=True, specular=True, background=(0.1, 0.11, 0.13)):
    """Lite shading descriptor.  colors: [(rgb, position, glossiness, ior)];
    lights: [(type, position_or_direction, rgb, brightness)]."""
    d = nd_lite_desc()
    d.color_count, d.light_count = len(colors), len(lights)
    d.ambient_occlusion, d.specular = int(bool(ambient_occlusion)), int(bool(specular))
    d.background[:] = [float(x) for x in background]
    for i, (rgb, pos, gloss, ior) in enumerate(colors):
        c = d.colors[i]
        c.color[:] = [float(x) for x in rgb]
        c.position, c.glossiness, c.ior = pos, gloss, ior
    for i, (kind, p, rgb, bright) in enumerate(lights):
        l = d.lights[i]
        l.type = kind
        l.position_or_direction[:] = [float(x) for x in p]
        l.color[:] = [float(x) for x in rgb]
        l.brightness = bright
    return d


class nd_gbuffer(C.Structure):
    _fields_ = [("depth", C.c_void_p), ("normal", C.c_void_p), ("trap", C.c_void_p), ("steps", C.c_void_p),
                ("iters", C.c_void_p), ("shade", C.c_void_p), ("shadow", C.c_void_p), ("depth64", C.c_void_p),
                ("evals", C.c_void_p), ("normal_half", C.c_void_p)]


class nd_march_opts(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("block", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("refill_threshold", C.c_int32), ("de_precision", C.c_int32), ("watchdog_ms", C.c_int32),
                ("accel_chain", C.c_int32), ("reserved", C.c_int32)]


class nd_stats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("de_evals", C.c_uint64), ("march_evals", C.c_uint64),
                ("normal_evals", C.c_uint64), ("shadow_evals", C.c_uint64), ("trap_evals", C.c_uint64),
                ("hits", C.c_uint64),
                ("refills", C.c_uint64), ("timeouts", C.c_uint32), ("kernel", C.c_uint32),
                ("march_ms", C.c_double), ("shade_ms", C.c_double), ("accel_voxels", C.c_uint64),
                ("accel_ms", C.c_double)]


class nd_tune_result(C.Structure):
    _fields_ = [("block", C.c_int32), ("blocks_per_sm", C.c_int32), ("refill_threshold", C.c_int32),
                ("kernel", C.c_int32), ("rays_per_s", C.c_double)]


class nd_orbit_camera(C.Structure):
    _fields_ = [("target", C.c_double * 3), ("yaw", C.c_double), ("pitch", C.c_double), ("dist", C.c_double),
                ("world_up", C.c_double * 3), ("fov_y_deg", C.c_double)]


def orbit_camera(yaw=0.0, pitch=0.0, dist=2.5, target=(0.0, 0.0, 0.0), world_up=(0.0, 1.0, 0.0),
                 fov_y_deg=60.0) -> nd_orbit_camera:
    """An orbit pose (angles in radians); nd_orbit_view turns it into a camera."""
    c = nd_orbit_camera()
    c.target[:] = [float(x) for x in target]
    c.yaw, c.pitch, c.dist = float(yaw), float(pitch), float(dist)
    c.world_up[:] = [float(x) for x in world_up]
    c.fov_y_deg = float(fov_y_deg)
    return c


def _sub(a, b):
    return [a[i] - b[i] for i in range(3)]


def _cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _norm(a):
    n = math.sqrt(sum(x * x for x in a))
    return [x / n for x in a]


def look_at(pos, target=(0.0, 0.0, 0.0), world_up=(0.0, 1.0, 0.0), fov_y_deg=60.0):
    """Camera basis as FreeCamera builds it (src/app/camera.zig:98-112):
    forward = normalize(target - pos), right = normalize(forward x up),
    up = normalize(right x forward); right and up are then scaled by tan(fov/2)
    (the reference has no FOV knob: |up| = 1 is a 90 degree vertical FOV)."""
    f = _norm(_sub(target, pos))
    r = _norm(_cross(f, list(world_up)))
    u = _norm(_cross(r, f))
    s = math.tan(math.radians(fov_y_deg) * 0.5)
    return f, [x * s for x in r], [x * s for x in u]


def make_view(formula: int, width: int, height: int, cam_pos, target=(0.0, 0.0, 0.0), fov_y_deg=60.0,
              params=None, world_up=(0.0, 1.0, 0.0), **kw) -> nd_view_desc:
    """A view with the reference's render defaults (RenderSettingsState and
    MarchPrecision, src/app/render_precision.zig:3-30: max_steps 256, max_dist 24,
    epsilon 5e-4 * t + 5e-5, refine_fast 4), overridable by keyword."""
    v = nd_view_desc()
    v.cam_pos[:] = [float(x) for x in cam_pos]
    f, r, u = look_at(list(cam_pos), list(target), world_up, fov_y_deg)
    v.fwd[:] = f
    v.right[:] = r
    v.up[:] = u
    v.width, v.height = width, height
    v.tile_x, v.tile_y, v.tile_w, v.tile_h = 0, 0, width, height
    v.formula = formula
    v.spp = 1
    v.seed = 0
    if params is not None:
        for i, p in enumerate(params[:ND_MAX_PARAMS]):
            v.params[i] = p
    v.trap.shape = ND_TRAP_POINT
    v.trap.mode = ND_TRAP_MIN
    v.trap.radius = 1.0
    v.trap.box[:] = [1.0, 1.0, 1.0]
    v.trap.span = 1.5
    v.max_steps = 256
    v.max_dist = 24.0
    v.eps_coef = 5e-4
    v.eps_floor = 5e-5
    v.refine_budget = 4
    v.march_verify = 0
    v.high_quality = 0
    v.hq_footprint_px = 2.0
    v.normal_mode = ND_NORMAL_TETRA
    v.normal_h_coef = 0.0
    v.shadow = 0
    v.shadow_k = 16.0
    v.step_safety = 1.0
    v.accel_res = 0          # empty-space accelerator off; the reference's defaults otherwise
    v.accel_levels = 6
    v.accel_safety = 0.92
    for k, val in kw.items():
        if k == "trap":
            for tk, tv in val.items():
                if isinstance(tv, (list, tuple)):
                    getattr(v.trap, tk)[:] = tv
                else:
                    setattr(v.trap, tk, tv)
        elif isinstance(val, (list, tuple)):
            getattr(v, k)[:] = list(val)
        else:
            setattr(v, k, val)
    return v


def rays_of(v: nd_view_desc) -> int:
    return int(v.spp) * int(v.tile_w) * int(v.tile_h)
