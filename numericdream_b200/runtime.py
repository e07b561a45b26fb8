"""Python host side over the C ABI (include/nd_march.h), through ctypes.

This mirrors the reference's host interface for the sphere-tracing path:

* ``FractalRenderer.rebuild(sources)`` stands where the reference's
  ``FractalRenderer.rebuild`` (src/gpu/fractal_renderer.zig:2927) compiles a scene's
  formula sources and stamps formula codes (``stampFormulaCodes``, :2882); errors are
  raised as ``FormulaError`` carrying the message the reference would copy into
  ``FormulaState.formula_error`` (src/app/formula.zig:73-77).
* ``FractalRenderer.render(views)`` stands where ``renderToImage`` (:3548) marches
  every pixel; it returns the G-buffer as torch tensors on the device.

torch is used only for device memory and streams.  The library is the in-tree
``libnd_march.so``; importing this module on a machine without it raises at once
(there is no CPU fallback).
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnd_march.so")

# every entry point include/nd_march.h declares, with its ctypes signature
_SIGNATURES = {
    "nd_abi_version": (C.c_int32, []),
    "nd_status_string": (C.c_char_p, [C.c_int32]),
    "nd_formula_count": (C.c_int32, [C.POINTER(C.c_int32)]),
    "nd_formula_find": (C.c_int32, [C.c_char_p, C.POINTER(C.c_int32)]),
    "nd_formula_name": (C.c_int32, [C.c_int32, C.c_char_p, C.c_size_t]),
    "nd_formula_register": (C.c_int32, [C.c_char_p, C.c_size_t, C.POINTER(C.c_int32), C.c_char_p, C.c_size_t]),
    "nd_formula_params": (C.c_int32, [C.c_int32, C.POINTER(abi.nd_param_info), C.POINTER(C.c_int32)]),
    "nd_view_defaults": (C.c_int32, [C.c_int32, C.POINTER(abi.nd_view_desc)]),
    "nd_ctx_create": (C.c_int32, [C.c_int32, C.POINTER(C.c_void_p)]),
    "nd_ctx_destroy": (C.c_int32, [C.c_void_p]),
    "nd_last_error": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "nd_last_stats": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_stats)]),
    "nd_count_rays": (C.c_int32, [C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(C.c_int64)]),
    "nd_march_forward": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32,
                                     C.POINTER(abi.nd_march_opts), C.POINTER(abi.nd_gbuffer), C.c_void_p]),
    "nd_autotune": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(abi.nd_gbuffer),
                                C.POINTER(abi.nd_tune_result)]),
    "nd_graph_capture": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32,
                                     C.POINTER(abi.nd_march_opts), C.POINTER(abi.nd_gbuffer), C.c_void_p,
                                     C.POINTER(C.c_void_p)]),
    "nd_graph_capture_scenes": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32,
                                            C.POINTER(C.c_int32), C.POINTER(abi.nd_scene_desc), C.c_int32,
                                            C.POINTER(abi.nd_march_opts), C.POINTER(abi.nd_gbuffer), C.c_void_p,
                                            C.POINTER(C.c_void_p)]),
    "nd_image_prepare": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]),
    "nd_tune_cache_save": (C.c_int32, [C.c_char_p]),
    "nd_tune_cache_load": (C.c_int32, [C.c_char_p, C.POINTER(C.c_int32)]),
    "nd_graph_launch": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "nd_graph_destroy": (C.c_int32, [C.c_void_p]),
    "nd_sizeof": (C.c_size_t, [C.c_char_p]),
    "nd_de_points": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int64, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "nd_orbit_view": (C.c_int32, [C.POINTER(abi.nd_orbit_camera), C.POINTER(abi.nd_view_desc)]),
    "nd_accel_grid": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32, C.c_void_p, C.c_int64,
                                  C.c_void_p, C.POINTER(C.c_int64)]),
    "nd_scene_file_load": (C.c_int32, [C.c_char_p, C.c_size_t, C.c_int32, C.c_int32, C.POINTER(abi.nd_view_desc),
                                       C.POINTER(abi.nd_scene_desc), C.POINTER(C.c_int32), C.c_char_p, C.c_size_t]),
    "nd_shade_lite": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(abi.nd_lite_desc),
                                  C.POINTER(abi.nd_gbuffer), C.c_void_p, C.c_void_p]),
    "nd_scene_file_lite": (C.c_int32, [C.c_char_p, C.c_size_t, C.c_int32, C.POINTER(abi.nd_lite_desc), C.c_char_p,
                                       C.c_size_t]),
    "nd_shade_lite_scenes": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(C.c_int32),
                                         C.POINTER(abi.nd_scene_desc), C.c_int32, C.POINTER(abi.nd_lite_desc),
                                         C.POINTER(abi.nd_lite_desc), C.POINTER(abi.nd_gbuffer), C.c_void_p,
                                         C.c_void_p]),
    "nd_measure_fp32_peak": (C.c_int32, [C.c_void_p, C.c_double, C.POINTER(C.c_double)]),
    "nd_march_forward_scenes": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(C.c_int32),
                                            C.POINTER(abi.nd_scene_desc), C.c_int32, C.POINTER(abi.nd_march_opts),
                                            C.POINTER(abi.nd_gbuffer), C.c_void_p]),
    "nd_march_forward_noalloc": (C.c_int32, [C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(abi.nd_march_opts),
                                             C.POINTER(abi.nd_gbuffer), C.c_void_p]),
    "nd_march_forward_noalloc_stats": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_stats), C.c_char_p, C.c_size_t]),
    "nd_march_backward": (C.c_int32, [C.c_void_p, C.POINTER(abi.nd_view_desc), C.POINTER(abi.nd_orbit_camera),
                                      C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(abi.nd_gbuffer),
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(abi.nd_march_opts),
                                      C.c_void_p]),
}

_lib = None


class NDError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        name = abi.STATUS_NAMES[status] if 0 <= status < len(abi.STATUS_NAMES) else f"status {status}"
        super().__init__(f"{name}: {msg}" if msg else name)
        self.status = status


class FormulaError(NDError):
    """A formula source the library cannot use (the reference's formula_error text)."""


def load_library(path: str = LIB_PATH):
    """Load libnd_march.so (built in-tree by numericdream_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m numericdream_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check_layout(lib=None):
    """Compare the ctypes structure sizes with the library's own."""
    lib = lib or load_library()
    for name in ("nd_view_desc", "nd_trap_desc", "nd_gbuffer", "nd_march_opts", "nd_stats", "nd_param_info",
                 "nd_tune_result", "nd_orbit_camera", "nd_scene_desc", "nd_instance_desc", "nd_mixin_desc",
                 "nd_lite_desc", "nd_color_stop", "nd_light"):
        mine = C.sizeof(getattr(abi, name))
        theirs = lib.nd_sizeof(name.encode())
        if mine != theirs:
            raise AssertionError(f"{name}: ctypes size {mine} != C size {theirs}")


def formula_count() -> int:
    n = C.c_int32()
    load_library().nd_formula_count(C.byref(n))
    return n.value


def formula_name(fid: int) -> str:
    buf = C.create_string_buffer(64)
    st = load_library().nd_formula_name(fid, buf, 64)
    if st != abi.ND_OK:
        raise NDError(st, f"formula id {fid}")
    return buf.value.decode()


def formula_names() -> list:
    return [formula_name(i) for i in range(formula_count())]


def find_formula(name: str) -> int:
    out = C.c_int32()
    st = load_library().nd_formula_find(name.encode(), C.byref(out))
    if st != abi.ND_OK:
        raise NDError(st, f"formula {name!r} is not in this build")
    return out.value


def register_formula(source: str) -> int:
    out = C.c_int32()
    err = C.create_string_buffer(512)
    data = source.encode("utf-8")
    st = load_library().nd_formula_register(data, len(data), C.byref(out), err, 512)
    if st != abi.ND_OK:
        raise FormulaError(st, err.value.decode())
    return out.value


def prepare_image(rgba):
    """nd_image_prepare: a formula image's texels (uint32, 4 per texel) and per-channel
    slope bound from rgba, a (height, width, 4) float array of R, G, B premultiplied by
    alpha and alpha in [0, 1]."""
    import numpy as np

    a = np.ascontiguousarray(rgba, dtype=np.float32)
    if a.ndim != 3 or a.shape[2] != 4:
        raise ValueError("rgba must be (height, width, 4)")
    h, w = a.shape[:2]
    texels = np.zeros(h * w * 4, dtype=np.uint32)
    slope = np.zeros(4, dtype=np.float32)
    st = load_library().nd_image_prepare(a.ctypes.data, w, h, texels.ctypes.data, slope.ctypes.data)
    if st != abi.ND_OK:
        raise NDError(st, f"nd_image_prepare({w}x{h})")
    return texels, slope


def formula_params(fid: int) -> list:
    n = C.c_int32()
    buf = (abi.nd_param_info * abi.ND_MAX_PARAMS)()
    st = load_library().nd_formula_params(fid, buf, C.byref(n))
    if st != abi.ND_OK:
        raise NDError(st, f"formula id {fid}")
    return [buf[i] for i in range(n.value)]


def load_scene_file(source, width: int = 0, height: int = 0):
    """nd_scene_file_load: a .dream scene (a path or the JSON text) as (view, scene);
    scene is None when the view alone describes it (render with Context.forward),
    else render with Context.forward_scenes([view], [0], [scene], ...)."""
    if isinstance(source, (bytes, bytearray)):
        data = bytes(source)
    elif isinstance(source, str) and source.lstrip().startswith("{"):
        data = source.encode("utf-8")
    else:
        with open(source, "rb") as fh:
            data = fh.read()
    view, scene, needs = abi.nd_view_desc(), abi.nd_scene_desc(), C.c_int32()
    err = C.create_string_buffer(512)
    st = load_library().nd_scene_file_load(data, len(data), width, height, C.byref(view), C.byref(scene),
                                           C.byref(needs), err, 512)
    if st != abi.ND_OK:
        raise NDError(st, err.value.decode())
    return view, (scene if needs.value else None)


def load_scene_file_lite(source, instance: int = 0) -> abi.nd_lite_desc:
    """nd_scene_file_lite: the lite-shading descriptor (colour stops of one instance,
    point and global lights) of a .dream scene (a path or the JSON text)."""
    if isinstance(source, (bytes, bytearray)):
        data = bytes(source)
    elif isinstance(source, str) and source.lstrip().startswith("{"):
        data = source.encode("utf-8")
    else:
        with open(source, "rb") as fh:
            data = fh.read()
    lite = abi.nd_lite_desc()
    err = C.create_string_buffer(256)
    st = load_library().nd_scene_file_lite(data, len(data), instance, C.byref(lite), err, 256)
    if st != abi.ND_OK:
        raise NDError(st, err.value.decode())
    return lite


def view_defaults(fid: int) -> abi.nd_view_desc:
    v = abi.nd_view_desc()
    st = load_library().nd_view_defaults(fid, C.byref(v))
    if st != abi.ND_OK:
        raise NDError(st)
    return v


def orbit_view(cam: abi.nd_orbit_camera, view: abi.nd_view_desc) -> abi.nd_view_desc:
    """Set view's camera from an orbit pose (nd_orbit_view)."""
    st = load_library().nd_orbit_view(C.byref(cam), C.byref(view))
    if st != abi.ND_OK:
        raise NDError(st, "nd_orbit_view")
    return view


def total_rays(views) -> int:
    arr = (abi.nd_view_desc * len(views))(*views)
    t = C.c_int64()
    st = load_library().nd_count_rays(arr, len(views), C.byref(t))
    if st != abi.ND_OK:
        raise NDError(st)
    return t.value


@dataclass
class GBuffer:
    """Device G-buffer (torch tensors) for one forward call."""

    depth: "object"
    normal: "object" = None
    trap: "object" = None
    steps: "object" = None
    iters: "object" = None
    shade: "object" = None
    shadow: "object" = None
    depth64: "object" = None
    evals: "object" = None
    normal_half: "object" = None  # (n, 4) float16: the reference's RGBA16F normal target

    @staticmethod
    def allocate(n: int, device="cuda", full: bool = True) -> "GBuffer":
        import torch

        g = GBuffer(depth=torch.empty(n, dtype=torch.float32, device=device))
        if full:
            g.normal = torch.empty((n, 4), dtype=torch.float32, device=device)
            g.trap = torch.empty(n, dtype=torch.float32, device=device)
            g.steps = torch.empty(n, dtype=torch.int32, device=device)
            g.iters = torch.empty(n, dtype=torch.int32, device=device)
            g.shade = torch.empty(n, dtype=torch.float32, device=device)
            g.shadow = torch.empty(n, dtype=torch.float32, device=device)
            g.depth64 = torch.empty(n, dtype=torch.float64, device=device)
            g.evals = torch.empty(n, dtype=torch.int32, device=device)
        return g

    def as_abi(self) -> abi.nd_gbuffer:
        g = abi.nd_gbuffer()
        for f in ("depth", "normal", "trap", "steps", "iters", "shade", "shadow", "depth64", "evals", "normal_half"):
            t = getattr(self, f)
            setattr(g, f, None if t is None else t.data_ptr())
        return g

    def numpy(self) -> dict:
        out = {}
        for f in ("depth", "normal", "trap", "steps", "iters", "shade", "shadow", "depth64", "evals", "normal_half"):
            t = getattr(self, f)
            if t is not None:
                out[f] = t.cpu().numpy()
        return out


def make_opts(kernel=abi.ND_KERNEL_AUTO, blocks_per_sm=0, refill_threshold=0, de_precision=32, watchdog_ms=0,
              accel_chain=0, block=0):
    o = abi.nd_march_opts()
    o.kernel, o.blocks_per_sm, o.refill_threshold, o.block = kernel, blocks_per_sm, refill_threshold, block
    o.de_precision, o.watchdog_ms, o.accel_chain = de_precision, watchdog_ms, accel_chain
    return o


class Context:
    """One nd_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        self.device = device
        h = C.c_void_p()
        st = self.lib.nd_ctx_create(device, C.byref(h))
        if st != abi.ND_OK:
            raise NDError(st, f"nd_ctx_create(device={device})")
        self.handle = h

    def close(self):
        if self.handle:
            self.lib.nd_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        buf = C.create_string_buffer(512)
        self.lib.nd_last_error(self.handle, buf, 512)
        return buf.value.decode()

    def _check(self, st, what):
        if st != abi.ND_OK:
            raise NDError(st, f"{what}: {self.last_error()}")

    def forward(self, views, gbuf: GBuffer, opts: abi.nd_march_opts | None = None, stream=None):
        arr = (abi.nd_view_desc * len(views))(*views)
        g = gbuf.as_abi()
        s = None if stream is None else C.c_void_p(stream)
        st = self.lib.nd_march_forward(self.handle, arr, len(views), C.byref(opts) if opts is not None else None,
                                       C.byref(g), s)
        self._check(st, "nd_march_forward")

    def forward_scenes(self, views, view_scene, scenes, gbuf: GBuffer, opts: abi.nd_march_opts | None = None,
                       stream=None):
        """nd_march_forward_scenes: view i uses scenes[view_scene[i]] (-1: its own instance)."""
        arr = (abi.nd_view_desc * len(views))(*views)
        vs = (C.c_int32 * len(views))(*view_scene)
        sarr = (abi.nd_scene_desc * max(1, len(scenes)))(*scenes)
        g = gbuf.as_abi()
        s = None if stream is None else C.c_void_p(stream)
        st = self.lib.nd_march_forward_scenes(self.handle, arr, len(views), vs, sarr, len(scenes),
                                              C.byref(opts) if opts is not None else None, C.byref(g), s)
        self._check(st, "nd_march_forward_scenes")

    def backward(self, views, cams, gbuf: GBuffer, dL_dshade=None, param_idx=(), de_precision=32,
                 per_ray=False, stream=None):
        """dLoss/dtheta (nviews x (len(param_idx) + 3): params, yaw, pitch, dist) for
        dLoss/dshade (torch float32 on the device, one per ray).  With per_ray=True
        returns (grad or None, dshade/dtheta per ray: rays x (len(param_idx) + 3))."""
        import torch

        k = len(param_idx) + 3
        dev = gbuf.depth.device
        grad = torch.zeros((len(views), k), dtype=torch.float64, device=dev) if dL_dshade is not None else None
        per = torch.zeros((gbuf.depth.numel(), k), dtype=torch.float64, device=dev) if per_ray else None
        arr = (abi.nd_view_desc * len(views))(*views)
        carr = (abi.nd_orbit_camera * len(cams))(*cams)
        pidx = (C.c_int32 * max(1, len(param_idx)))(*param_idx)
        g = gbuf.as_abi()
        opts = make_opts(de_precision=de_precision)
        s = None if stream is None else C.c_void_p(stream)
        dl = dL_dshade.contiguous() if dL_dshade is not None else None
        st = self.lib.nd_march_backward(self.handle, arr, carr, len(views), pidx, len(param_idx), C.byref(g),
                                        dl.data_ptr() if dl is not None else None,
                                        grad.data_ptr() if grad is not None else None,
                                        per.data_ptr() if per is not None else None, C.byref(opts), s)
        self._check(st, "nd_march_backward")
        return (grad, per) if per_ray else grad

    def de_points(self, view: abi.nd_view_desc, pts, de_precision: int = 32):
        """DE, trap and changed-iteration count of view's formula at points (torch, on device)."""
        import torch

        pts = torch.as_tensor(pts, dtype=torch.float64).reshape(-1, 3).contiguous().to(f"cuda:{self.device}")
        n = pts.shape[0]
        de = torch.empty(n, dtype=torch.float64, device=pts.device)
        tr = torch.empty(n, dtype=torch.float64, device=pts.device)
        it = torch.empty(n, dtype=torch.int32, device=pts.device)
        st = self.lib.nd_de_points(self.handle, C.byref(view), n, pts.data_ptr(), de.data_ptr(), tr.data_ptr(),
                                   it.data_ptr(), de_precision, None)
        self._check(st, "nd_de_points")
        torch.cuda.synchronize(pts.device)
        return de.cpu().numpy(), tr.cpu().numpy(), it.cpu().numpy()

    def shade_lite(self, views, lites, gbuf: GBuffer, stream=None):
        """nd_shade_lite over the G-buffer of a forward of the same views: an (n, 4)
        float32 device tensor, rgb and w = 1 on a hit."""
        import torch

        n = gbuf.depth.shape[0]
        rgba = torch.empty((n, 4), dtype=torch.float32, device=gbuf.depth.device)
        arr = (abi.nd_view_desc * len(views))(*views)
        la = (abi.nd_lite_desc * len(views))(*lites)
        g = gbuf.as_abi()
        s = None if stream is None else C.c_void_p(stream)
        st = self.lib.nd_shade_lite(self.handle, arr, len(views), la, C.byref(g), rgba.data_ptr(), s)
        self._check(st, "nd_shade_lite")
        return rgba

    def shade_lite_scenes(self, views, view_scene, scenes, lites, instance_colors, gbuf: GBuffer, stream=None):
        """nd_shade_lite_scenes: instance_colors is one list of ND_MAX_INSTANCES
        descriptors per scene (shorter lists are padded with empty descriptors)."""
        import torch

        n = gbuf.depth.shape[0]
        rgba = torch.empty((n, 4), dtype=torch.float32, device=gbuf.depth.device)
        arr = (abi.nd_view_desc * len(views))(*views)
        vs = (C.c_int32 * len(views))(*view_scene)
        sarr = (abi.nd_scene_desc * max(1, len(scenes)))(*scenes)
        la = (abi.nd_lite_desc * len(views))(*lites)
        flat = []
        for per in instance_colors:
            flat += list(per) + [abi.nd_lite_desc()] * (abi.ND_MAX_INSTANCES - len(per))
        ic = (abi.nd_lite_desc * max(1, len(flat)))(*flat)
        g = gbuf.as_abi()
        s = None if stream is None else C.c_void_p(stream)
        st = self.lib.nd_shade_lite_scenes(self.handle, arr, len(views), vs, sarr, len(scenes), la, ic, C.byref(g),
                                           rgba.data_ptr(), s)
        self._check(st, "nd_shade_lite_scenes")
        return rgba

    def accel_grid(self, view: abi.nd_view_desc, de_precision: int = 32):
        """nd_accel_grid: the view's accelerator grid ([level][z][y][x], numpy) and its
        cascade placement (8 x (corner xyz, cell))."""
        import numpy as np
        import torch

        res = min(max(view.accel_res, 16), 160) // 4 * 4
        levels = min(max(view.accel_levels, 1), 8)
        grid = torch.empty(levels * res ** 3, dtype=torch.float32, device=f"cuda:{self.device}")
        prm = np.zeros((8, 4), np.float32)
        n = C.c_int64()
        st = self.lib.nd_accel_grid(self.handle, C.byref(view), de_precision, grid.data_ptr(), grid.numel(),
                                    prm.ctypes.data, C.byref(n))
        self._check(st, "nd_accel_grid")
        return grid.cpu().numpy().reshape(levels, res, res, res), prm

    def measure_fp32_peak(self, ms: float = 20.0) -> float:
        """nd_measure_fp32_peak: the device's FP32 FMA throughput in TFLOP/s."""
        out = C.c_double()
        st = self.lib.nd_measure_fp32_peak(self.handle, ms, C.byref(out))
        self._check(st, "nd_measure_fp32_peak")
        return out.value

    def stats(self) -> abi.nd_stats:
        out = abi.nd_stats()
        st = self.lib.nd_last_stats(self.handle, C.byref(out))
        self._check(st, "nd_last_stats")
        return out

    def autotune(self, views, scratch: GBuffer) -> abi.nd_tune_result:
        arr = (abi.nd_view_desc * len(views))(*views)
        g = scratch.as_abi()
        r = abi.nd_tune_result()
        st = self.lib.nd_autotune(self.handle, arr, len(views), C.byref(g), C.byref(r))
        self._check(st, "nd_autotune")
        return r

    @staticmethod
    def tune_cache_save(path: str):
        """nd_tune_cache_save: the autotuner's winners (every context, every GPU) to a JSON file."""
        st = load_library().nd_tune_cache_save(path.encode())
        if st != abi.ND_OK:
            raise NDError(st, f"nd_tune_cache_save({path!r})")

    @staticmethod
    def tune_cache_load(path: str) -> int:
        """nd_tune_cache_load: read winners saved earlier; returns the entries read."""
        n = C.c_int32()
        st = load_library().nd_tune_cache_load(path.encode(), C.byref(n))
        if st != abi.ND_OK:
            raise NDError(st, f"nd_tune_cache_load({path!r})")
        return n.value

    def capture(self, views, gbuf: GBuffer, opts=None, stream=None) -> "Graph":
        arr = (abi.nd_view_desc * len(views))(*views)
        g = gbuf.as_abi()
        h = C.c_void_p()
        s = None if stream is None else C.c_void_p(stream)
        st = self.lib.nd_graph_capture(self.handle, arr, len(views), C.byref(opts) if opts is not None else None,
                                       C.byref(g), s, C.byref(h))
        self._check(st, "nd_graph_capture")
        return Graph(self, h)

    def capture_scenes(self, views, view_scene, scenes, gbuf: GBuffer, opts=None, stream=None) -> "Graph":
        """nd_graph_capture_scenes: a graph of forward_scenes(views, view_scene, scenes)."""
        arr = (abi.nd_view_desc * len(views))(*views)
        vs = (C.c_int32 * len(views))(*view_scene)
        sarr = (abi.nd_scene_desc * max(1, len(scenes)))(*scenes)
        g = gbuf.as_abi()
        h = C.c_void_p()
        s = None if stream is None else C.c_void_p(stream)
        st = self.lib.nd_graph_capture_scenes(self.handle, arr, len(views), vs, sarr, len(scenes),
                                              C.byref(opts) if opts is not None else None, C.byref(g), s,
                                              C.byref(h))
        self._check(st, "nd_graph_capture_scenes")
        return Graph(self, h)


class Graph:
    def __init__(self, ctx: Context, handle):
        self.ctx, self.handle = ctx, handle

    def launch(self, stream=None):
        s = None if stream is None else C.c_void_p(stream)
        st = self.ctx.lib.nd_graph_launch(self.handle, s)
        self.ctx._check(st, "nd_graph_launch")

    def close(self):
        if self.handle:
            self.ctx.lib.nd_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class FractalRenderer:
    """The reference's renderer surface for this path (rebuild + render)."""

    def __init__(self, device: int = 0):
        self.ctx = Context(device)
        self.codes: list = []

    def rebuild(self, sources) -> list:
        """Register each formula source (WGSL text) or built-in name; returns codes."""
        codes = []
        for s in sources:
            if "\n" in s or "fn " in s:
                codes.append(register_formula(s))
            else:
                codes.append(find_formula(s))
        self.codes = codes
        return codes

    def render(self, views, opts=None, full: bool = True, stream=None) -> GBuffer:
        import torch

        n = total_rays(views)
        g = GBuffer.allocate(n, device=torch.device("cuda", self.ctx.device), full=full)
        self.ctx.forward(views, g, opts, stream=stream)
        return g

    def render_to_image(self, scene_file, width: int = 0, height: int = 0) -> bytes:
        """renderToImage (fractal_renderer.zig:3548) for this pass: a .dream scene's
        geometry and lite colour as width x height RGBA8 (colour clamped to [0, 1];
        the reference's tone mapping and post effects are not part of this pass)."""
        import numpy as np

        from .render import render_scene_file

        img, _ = render_scene_file(self.ctx, scene_file, width, height)
        rgba = np.empty(img.shape, np.uint8)
        rgba[..., :3] = (np.clip(img[..., :3], 0.0, 1.0) * 255.0 + 0.5).astype(np.uint8)
        rgba[..., 3] = 255
        return rgba.tobytes()
