"""ctypes front end of the CPU oracle (test infrastructure only; see oracle.hpp)."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from numericdream_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_LIB_FMA = None


def lib(fma: bool = False):
    """The oracle library; fma=True: the same code compiled with fused multiply-adds."""
    global _LIB, _LIB_FMA
    from . import build_oracle

    if fma:
        if _LIB_FMA is None:
            _LIB_FMA = _setup(C.CDLL(build_oracle.build(fma=True)))
        return _LIB_FMA
    if _LIB is None:
        _LIB = _setup(C.CDLL(build_oracle.build()))  # rebuilt only when a source is newer than the library
    return _LIB


def _setup(L):
    L.oracle_formula_index.argtypes = [C.c_char_p]
    L.oracle_de.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_void_p]
    L.oracle_render.argtypes = ([C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_int64, C.c_int64] + [C.c_void_p] * 10
                                + [C.c_double])
    L.oracle_render_scene.argtypes = ([C.c_void_p] * 4 + [C.c_int, C.c_int, C.c_int64, C.c_int64]
                                      + [C.c_void_p] * 10 + [C.c_double])
    L.oracle_scene_de.argtypes = ([C.c_void_p] * 3 + [C.c_double, C.c_int, C.c_int64] + [C.c_void_p] * 4)
    L.oracle_accel_grid.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_int64,
                                       C.c_void_p]
    L.oracle_accel_grid.restype = C.c_int64
    L.oracle_march_dirs.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p]
    L.oracle_combine.argtypes = [C.c_int64] + [C.c_void_p] * 5
    L.oracle_shade_lite.argtypes = ([C.c_void_p, C.c_char_p, C.c_void_p, C.c_int, C.c_int64, C.c_int64]
                                       + [C.c_void_p] * 4)
    L.oracle_ao.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int64] + [C.c_void_p] * 4
    L.oracle_strip_fresnel.argtypes = [C.c_int64] + [C.c_void_p] * 6
    L.oracle_shade_lite_scene.argtypes = ([C.c_void_p] * 6 + [C.c_int, C.c_int64, C.c_int64]
                                             + [C.c_void_p] * 4)
    L.oracle_combine_weight.argtypes = [C.c_int64] + [C.c_void_p] * 5
    L.oracle_max_threads.restype = C.c_int
    L.oracle_set_image.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]
    return L


def set_image(texels=None, width=0, height=0, slope=None):
    """The formula image `// @image` formulas read (texels as nd_image_prepare writes
    them: uint32, 4 per texel); None clears it.  Both oracle builds get it."""
    keep = []
    for fma in (False, True):
        if texels is None:
            lib(fma).oracle_set_image(None, 0, 0, None)
            continue
        t = np.ascontiguousarray(texels, dtype=np.uint32)
        sl = np.ascontiguousarray(slope, dtype=np.float32)
        keep += [t, sl]
        lib(fma).oracle_set_image(t.ctypes.data, int(width), int(height), sl.ctypes.data)


def has_formula(name: str) -> bool:
    return lib().oracle_formula_index(name.encode()) >= 0


def max_threads() -> int:
    return lib().oracle_max_threads()


def de(name: str, params, pts, precision=64, trap: abi.nd_trap_desc | None = None):
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    n = pts.shape[0]
    prm = np.zeros(16, np.float32)
    prm[: len(params)] = params
    out = np.zeros(n, np.float64)
    tr = np.zeros(n, np.float64)
    it = np.zeros(n, np.int32)
    rc = lib().oracle_de(name.encode(), prm.ctypes.data, C.addressof(trap) if trap is not None else None,
                         precision, n, pts.ctypes.data, out.ctypes.data, tr.ctypes.data, it.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle has no formula {name!r}")
    return out, tr, it


STABILITY_DELTA = 1e-4
_KEYS = ["depth", "normal", "trap", "steps", "iters", "shade", "shadow", "depth64", "evals", "margin"]


def _outputs(n):
    return {
        "depth": np.zeros(n, np.float32), "normal": np.zeros((n, 4), np.float32), "trap": np.zeros(n, np.float32),
        "steps": np.zeros(n, np.uint32), "iters": np.zeros(n, np.uint32), "shade": np.zeros(n, np.float32),
        "shadow": np.zeros(n, np.float32), "depth64": np.zeros(n, np.float64), "evals": np.zeros(n, np.uint32),
        "margin": np.zeros(n, np.float64),
    }


def render(view: abi.nd_view_desc, formula_name: str, precision=64, nthreads=0, first=0, n=None, de_scale=1.0,
           fma=False):
    """Trace rays [first, first+n) of one view; returns a dict of numpy arrays.  fma:
    with the oracle compiled with fused multiply-adds (differs by rounding only)."""
    total = abi.rays_of(view)
    if n is None:
        n = total - first
    out = _outputs(n)
    rc = lib(fma).oracle_render(C.addressof(view), formula_name.encode(), precision, nthreads, first, n,
                             *[out[k].ctypes.data for k in _KEYS], de_scale)
    if rc != 0:
        raise ValueError(f"oracle has no formula {formula_name!r}")
    return out




def unstable_rays(view: abi.nd_view_desc, formula_name: str, delta: float = STABILITY_DELTA, nthreads=0):
    """Rays whose FP64 outcome (hit/miss or probe-step count) changes when every DE
    value is scaled by 1 - delta or 1 + delta: their integer outputs are not
    determined at FP32 precision (the boundary-case policy)."""
    base = render(view, formula_name, 64, nthreads)
    lo = render(view, formula_name, 64, nthreads, de_scale=1.0 - delta)
    hi = render(view, formula_name, 64, nthreads, de_scale=1.0 + delta)
    h = [o["normal"][:, 3] > 0.5 for o in (base, lo, hi)]
    unstable = (h[0] != h[1]) | (h[0] != h[2])
    unstable |= (base["steps"] != lo["steps"]) | (base["steps"] != hi["steps"])
    return unstable, base


def _scene_kinds(scene: abi.nd_scene_desc, names):
    """Oracle formula kinds of a scene's instances and mixins; names maps a formula
    id to its formula name."""
    def kind(fid):
        k = lib().oracle_formula_index(names(fid).encode())
        if k < 0:
            raise ValueError(f"oracle has no formula {names(fid)!r}")
        return k

    kinds = np.zeros(abi.ND_MAX_INSTANCES, np.int32)
    mk = np.zeros((abi.ND_MAX_INSTANCES, abi.ND_MAX_MIXINS), np.int32)
    for i in range(scene.instance_count):
        inst = scene.instances[i]
        kinds[i] = kind(inst.formula)
        for j in range(inst.mixin_count):
            mk[i, j] = kind(inst.mixins[j].formula)
    return kinds, mk


def scene_de(scene: abi.nd_scene_desc, names, pts, max_dist=24.0, precision=64):
    """The scene DE, nearest instance's trap and changed-iteration count at points."""
    kinds, mk = _scene_kinds(scene, names)
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    n = pts.shape[0]
    out, tr, it = np.zeros(n, np.float64), np.zeros(n, np.float64), np.zeros(n, np.int32)
    rc = lib().oracle_scene_de(C.addressof(scene), kinds.ctypes.data, mk.ctypes.data, max_dist, precision, n,
                               pts.ctypes.data, out.ctypes.data, tr.ctypes.data, it.ctypes.data)
    if rc != 0:
        raise ValueError("oracle_scene_de refused the scene")
    return out, tr, it


def render_scene(view: abi.nd_view_desc, scene: abi.nd_scene_desc, names, precision=64, nthreads=0, first=0, n=None,
                 de_scale=1.0):
    """Trace rays of one view against a multi-instance scene; names maps a formula id
    to its formula name (the ids the instances and mixins use)."""
    kinds, mk = _scene_kinds(scene, names)
    total = abi.rays_of(view)
    if n is None:
        n = total - first
    out = _outputs(n)
    rc = lib().oracle_render_scene(C.addressof(view), C.addressof(scene), kinds.ctypes.data, mk.ctypes.data,
                                   precision, nthreads, first, n, *[out[k].ctypes.data for k in _KEYS], de_scale)
    if rc != 0:
        raise ValueError("oracle_render_scene refused the scene")
    return out


def unstable_scene_rays(view: abi.nd_view_desc, scene: abi.nd_scene_desc, names, delta: float = STABILITY_DELTA,
                        nthreads=0):
    """unstable_rays for a view rendered against a multi-instance scene."""
    base = render_scene(view, scene, names, 64, nthreads)
    lo = render_scene(view, scene, names, 64, nthreads, de_scale=1.0 - delta)
    hi = render_scene(view, scene, names, 64, nthreads, de_scale=1.0 + delta)
    h = [o["normal"][:, 3] > 0.5 for o in (base, lo, hi)]
    unstable = (h[0] != h[1]) | (h[0] != h[2])
    unstable |= (base["steps"] != lo["steps"]) | (base["steps"] != hi["steps"])
    return unstable, base


def accel_grid(view: abi.nd_view_desc, formula_name: str, precision=64, nthreads=0):
    """The view's empty-space accelerator grid ([level][z][y][x] safe skips) and its
    cascade placement (8 x (corner xyz, cell))."""
    res = min(max(view.accel_res, 16), 160) // 4 * 4
    levels = min(max(view.accel_levels, 1), 8)
    grid = np.zeros(levels * res ** 3, np.float32)
    prm = np.zeros((8, 4), np.float32)
    n = lib().oracle_accel_grid(C.addressof(view), formula_name.encode(), precision, nthreads, grid.ctypes.data,
                                grid.size, prm.ctypes.data)
    if n < 0:
        raise ValueError("oracle_accel_grid refused the view")
    return grid.reshape(levels, res, res, res), prm


def march_dirs(view: abi.nd_view_desc, formula_name: str, dirs, precision=64):
    """The oracle's primary march from the view's camera along given unit directions:
    (n, 4) array of hit, t, probe steps, DE evaluations."""
    dirs = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((dirs.shape[0], 4), np.float64)
    rc = lib().oracle_march_dirs(C.addressof(view), formula_name.encode(), precision, dirs.shape[0],
                                 dirs.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle has no formula {formula_name!r}")
    return out


def combine(mode, d, di, k):
    """The oracle's combine_de distance (f32) elementwise."""
    mode = np.ascontiguousarray(mode, np.int32)
    d, di, k = (np.ascontiguousarray(x, np.float32) for x in (d, di, k))
    out = np.zeros(mode.size, np.float32)
    lib().oracle_combine(mode.size, mode.ctypes.data, d.ctypes.data, di.ctypes.data, k.ctypes.data,
                         out.ctypes.data)
    return out


def shade_lite(view: abi.nd_view_desc, formula_name: str, lite: abi.nd_lite_desc, gbuf: dict, precision=64, first=0):
    """The oracle's lite shading from forward outputs (depth64, normal, trap arrays)."""
    depth64 = np.ascontiguousarray(gbuf["depth64"], np.float64)
    normal = np.ascontiguousarray(gbuf["normal"], np.float32)
    trap = np.ascontiguousarray(gbuf["trap"], np.float32)
    n = depth64.shape[0]
    out = np.zeros((n, 4), np.float32)
    rc = lib().oracle_shade_lite(C.addressof(view), formula_name.encode(), C.addressof(lite), precision, first, n,
                                 depth64.ctypes.data, normal.ctypes.data, trap.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"oracle has no formula {formula_name!r}")
    return out


def ao(view: abi.nd_view_desc, formula_name: str, pos, nrm, t, precision=64):
    """The oracle's calc_ao at hit points."""
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    nrm = np.ascontiguousarray(nrm, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(t, np.float64)
    out = np.zeros(t.size, np.float64)
    lib().oracle_ao(C.addressof(view), formula_name.encode(), precision, t.size, pos.ctypes.data, nrm.ctypes.data,
                    t.ctypes.data, out.ctypes.data)
    return out


def strip_fresnel(sor, v, cosv, ior):
    """The oracle's orbit_trap_to_strip (sor: (n, 3) span, offset, repeat) and fresnel_schlick, f32."""
    sor = np.ascontiguousarray(sor, np.float32).reshape(-1, 3)
    v, cosv, ior = (np.ascontiguousarray(x, np.float32) for x in (v, cosv, ior))
    st, fr = np.zeros(v.size, np.float32), np.zeros(v.size, np.float32)
    lib().oracle_strip_fresnel(v.size, sor.ctypes.data, v.ctypes.data, cosv.ctypes.data, ior.ctypes.data,
                               st.ctypes.data, fr.ctypes.data)
    return st, fr


def shade_lite_scene(view: abi.nd_view_desc, scene: abi.nd_scene_desc, names, lite: abi.nd_lite_desc, instance_colors,
                     gbuf: dict, precision=64, first=0):
    """The oracle's lite shading of a scene view from forward outputs; instance_colors:
    up to ND_MAX_INSTANCES descriptors (their colour stops, sorted by position)."""
    kinds, mk = _scene_kinds(scene, names)
    per = list(instance_colors) + [abi.nd_lite_desc()] * (abi.ND_MAX_INSTANCES - len(instance_colors))
    ic = (abi.nd_lite_desc * abi.ND_MAX_INSTANCES)(*per)
    depth64 = np.ascontiguousarray(gbuf["depth64"], np.float64)
    normal = np.ascontiguousarray(gbuf["normal"], np.float32)
    trap = np.ascontiguousarray(gbuf["trap"], np.float32)
    n = depth64.shape[0]
    out = np.zeros((n, 4), np.float32)
    rc = lib().oracle_shade_lite_scene(C.addressof(view), C.addressof(scene), kinds.ctypes.data, mk.ctypes.data,
                                       C.addressof(lite), C.addressof(ic), precision, first, n, depth64.ctypes.data,
                                       normal.ctypes.data, trap.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise ValueError("oracle_shade_lite_scene refused the scene")
    return out


def combine_weight(mode, d, di, k):
    """The oracle's combine_de material weight (f32) elementwise."""
    mode = np.ascontiguousarray(mode, np.int32)
    d, di, k = (np.ascontiguousarray(x, np.float32) for x in (d, di, k))
    out = np.zeros(mode.size, np.float32)
    lib().oracle_combine_weight(mode.size, mode.ctypes.data, d.ctypes.data, di.ctypes.data, k.ctypes.data,
                                out.ctypes.data)
    return out
