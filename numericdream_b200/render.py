"""A scene file to a colour image: the view, scene and lite shading descriptors of a
.dream file (nd_scene_file_load / nd_scene_file_lite), the forward march, and the
lite shading pass (nd_shade_lite / nd_shade_lite_scenes) — the geometry and lite
colour of the reference's render_lite path (template.wgsl:4446-4458) for one frame."""

from __future__ import annotations

import numpy as np

from . import abi, runtime


def render_scene_file(ctx: runtime.Context, source, width: int = 0, height: int = 0, opts=None, stream=None):
    """Render a .dream scene (path or JSON text) at width x height (0: the file's
    export size).  Returns (rgba, gbuf): an (height, width, 4) float32 array (w = hit)
    and the forward G-buffer as numpy arrays."""
    view, scene = runtime.load_scene_file(source, width, height)
    lite = runtime.load_scene_file_lite(source, 0)
    n = abi.rays_of(view)
    g = runtime.GBuffer.allocate(n)
    opts = opts or runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT)
    if scene is None:
        ctx.forward([view], g, opts, stream=stream)
        rgba = ctx.shade_lite([view], [lite], g, stream=stream)
    else:
        colors = [runtime.load_scene_file_lite(source, i) for i in range(scene.instance_count)]
        ctx.forward_scenes([view], [0], [scene], g, opts, stream=stream)
        rgba = ctx.shade_lite_scenes([view], [0], [scene], [lite], [colors], g, stream=stream)
    img = rgba.cpu().numpy().reshape(view.tile_h, view.tile_w, 4)
    return img, g.numpy()


def write_ppm(path: str, rgba) -> None:
    """An 8-bit binary PPM of an (h, w, 3+) float image (clamped to [0, 1])."""
    rgb = np.clip(np.asarray(rgba)[..., :3], 0.0, 1.0)
    h, w = rgb.shape[:2]
    with open(path, "wb") as fh:
        fh.write(f"P6 {w} {h} 255\n".encode())
        fh.write((rgb * 255.0 + 0.5).astype(np.uint8).tobytes())
