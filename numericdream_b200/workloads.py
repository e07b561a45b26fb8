"""Synthetic benchmark workloads for the sphere-tracing pass (seeded, no datasets).

Five workloads, each a list of ``nd_view_desc`` (see include/nd_march.h):

* ``mandelbulb_256``     Mandelbulb power 8, 12 iterations, bailout 2; 256x256 rays from
                        (0, 0, -2.5) at the origin, 60 deg FOV; max 256 steps, eps 1e-4 t;
                        central-difference normals h = 1e-4 t; sphere orbit trap.
* ``mandelbox_1080p``    Mandelbox scale -1.5, fold limit 1, min radius 0.5 (r^2 0.25),
                        fixed radius 1, 15 iterations; 1920x1080 x 4 jittered rays per
                        pixel; max 512 steps, eps 5e-5 t; one directional shadow ray per
                        hit, k = 16; box-shell orbit trap.
* ``batched_64``         64 views, sides log-uniform in [64, 1024], formulas drawn from
                        Mandelbulb (power U[4,10]), Mandelbox (scale U[-2,-1.2]), Menger
                        (3-6 iterations), pseudo-Kleinian (box size U[0.8,1.2]); cameras
                        on spheres of radius U[1.5,4] aimed at the origin; max 384 steps.
* ``mandelbulb_512``     the differentiation workload's view: Mandelbulb with the escape
                        radius as a parameter, Lambert shading from one light, orbit
                        camera; ``differentiation_16`` makes its 16 problems.
* ``deepzoom_4096``      Mandelbox scale -1.5, 30 iterations, 4096x4096 in 16 tiles of
                        1024x1024, FOV 0.01 deg, camera 1e-5 from the surface.

Values the workloads do not fix are the reference's render defaults
(src/app/render_precision.zig:3-30): max_dist 24, eps floor 5e-5 unless stated,
bisection refinement budget 4 (refine_fast), no verify pass.
"""

from __future__ import annotations

import math
import random

from . import abi

MANDELBULB = "mandelbrot"            # built-in formula (src/gpu/shaders/mandelbrot.wgsl)
MANDELBOX = "amazingbox_box"
MENGER = "menger3_ifs"
PSEUDO_KLEINIAN = "pseudokleinian_kleinian"
MANDELBULB_BAILOUT = "mandelbulb_bailout"   # this package's formulas/mandelbulb_bailout.wgsl

# default light of the shadowed workloads (unit direction TO the light)
LIGHT_DIR = (0.4, 0.8, -0.45)


def _ids(resolve):
    return {n: resolve(n) for n in (MANDELBULB, MANDELBOX, MENGER, PSEUDO_KLEINIAN)}


def mandelbox_params(scale=-1.5, iterations=15):
    # Scale, MinRadius, FixedRadius, FoldingLimit, Iterations, RotX/Y/Z, CScale, JuliaX/Y/Z
    return [scale, 0.5, 1.0, 1.0, float(iterations), 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0]


def mandelbulb_params(power=8.0, iterations=12):
    return [power, float(iterations)]


def menger_params(iterations=4):
    # Iterations, Scalex/y/z, Scale, RotX/Y/Z (formulas/menger3_ifs.wgsl defaults)
    return [float(iterations), 1.0, 1.0, 1.0, 3.0, 0.0, 0.0, 0.0]


def pseudo_kleinian_params(box_size=1.0):
    # CenterX/Y/Z, Radius, CellSize, Iterations, CScale, JuliaX/Y/Z.  "Box size" is
    # the lattice cube's half-width: CellSize = 2 * box size.
    return [1.0, 1.0, 1.0, 1.0, 2.0 * box_size, 14.0, 1.0, 0.0, 0.0, 0.0]


def mandelbulb_256(resolve, size=256):
    fid = resolve(MANDELBULB)
    v = abi.make_view(fid, size, size, (0.0, 0.0, -2.5), fov_y_deg=60.0, params=mandelbulb_params(8.0, 12),
                      max_steps=256, eps_coef=1e-4, eps_floor=0.0, normal_mode=abi.ND_NORMAL_CENTRAL,
                      normal_h_coef=1e-4, trap={"shape": abi.ND_TRAP_SPHERE, "radius": 1.0})
    return [v]


def reference_initial_camera():
    """FreeCamera.initial (src/app/camera.zig:98-107): yaw 0.7, pitch 0.35, distance 3.2."""
    yaw, pitch, dist = 0.7, 0.35, 3.2
    cp = math.cos(pitch)
    return (dist * cp * math.cos(yaw), dist * math.sin(pitch), dist * cp * math.sin(yaw))


def mandelbox_1080p(resolve, width=1920, height=1080, spp=4, seed=1234):
    fid = resolve(MANDELBOX)
    # the reference camera has no FOV knob: |up| = 1, a 90 degree vertical FOV
    v = abi.make_view(fid, width, height, reference_initial_camera(), fov_y_deg=90.0,
                      params=mandelbox_params(-1.5, 15), spp=spp, seed=seed, max_steps=512, eps_coef=5e-5,
                      eps_floor=0.0, normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=0.0, shadow=1,
                      light_dir=list(LIGHT_DIR), shadow_k=16.0,
                      trap={"shape": abi.ND_TRAP_BOX, "box": [1.0, 1.0, 1.0]})
    return [v]


def batched_64(resolve, nviews=64, seed=7, min_side=64, max_side=1024, max_steps=384):
    rng = random.Random(seed)
    ids = _ids(resolve)
    kinds = [MANDELBULB, MANDELBOX, MENGER, PSEUDO_KLEINIAN]
    views = []
    for i in range(nviews):
        w = int(round(math.exp(rng.uniform(math.log(min_side), math.log(max_side)))))
        h = int(round(math.exp(rng.uniform(math.log(min_side), math.log(max_side)))))
        kind = kinds[rng.randrange(4)]
        if kind == MANDELBULB:
            params = mandelbulb_params(rng.uniform(4.0, 10.0), 6)
        elif kind == MANDELBOX:
            params = mandelbox_params(rng.uniform(-2.0, -1.2), 12)
        elif kind == MENGER:
            params = menger_params(rng.randint(3, 6))
        else:
            params = pseudo_kleinian_params(rng.uniform(0.8, 1.2))
        # uniform direction on the sphere, radius U[1.5, 4]
        z = rng.uniform(-1.0, 1.0)
        phi = rng.uniform(0.0, 2.0 * math.pi)
        s = math.sqrt(max(0.0, 1.0 - z * z))
        r = rng.uniform(1.5, 4.0)
        pos = (r * s * math.cos(phi), r * s * math.sin(phi), r * z)
        up = (0.0, 1.0, 0.0) if abs(pos[1]) < 0.99 * r else (1.0, 0.0, 0.0)
        v = abi.make_view(ids[kind], w, h, pos, fov_y_deg=60.0, params=params, world_up=up,
                          max_steps=max_steps, normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=1e-4,
                          trap={"shape": abi.ND_TRAP_SPHERE, "radius": 1.0}, seed=seed * 1000 + i)
        views.append(v)
    return views


def mandelbulb_512(resolve, power=8.0, yaw=0.0, pitch=0.0, dist=2.5, size=512, bailout=2.0):
    """The differentiation workload's view: Mandelbulb (12 iterations, escape radius
    `bailout`, formulas/mandelbulb_bailout.wgsl of this package) with Lambert shading
    from one directional light, seen by an orbit camera (angles in radians) around
    the origin.  The hit is refined by a 40-step FP64 bisection on DE = eps(t) that
    runs to the end of its budget (ND_VIEW_EXACT_HIT), so the hit distance is a
    smooth function of theta.  Returns (view, orbit camera)."""
    from . import runtime

    fid = resolve(MANDELBULB_BAILOUT)
    cam = abi.orbit_camera(yaw=yaw, pitch=pitch, dist=dist, fov_y_deg=60.0)
    v = abi.make_view(fid, size, size, (0.0, 0.0, -dist), fov_y_deg=60.0, params=[power, 12.0, bailout],
                      max_steps=256, eps_coef=1e-4, eps_floor=0.0, refine_budget=40,
                      normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=1e-4, light_dir=list(LIGHT_DIR),
                      flags=abi.ND_VIEW_EXACT_HIT)
    runtime.orbit_view(cam, v)
    return v, cam


def differentiation_16(resolve, size=512, problems=16, seed=11):
    """16 problems: start power U[6,10] (seeded), bailout 2, camera yaw 0, pitch 0,
    distance 2.5; each target is rendered at power 8 with the camera yawed +2 degrees.
    Returns (start views, start cameras, target views, target cameras)."""
    rng = random.Random(seed)
    sv, sc, tv, tc = [], [], [], []
    for _ in range(problems):
        v, c = mandelbulb_512(resolve, power=rng.uniform(6.0, 10.0), size=size)
        sv.append(v)
        sc.append(c)
        v, c = mandelbulb_512(resolve, power=8.0, yaw=math.radians(2.0), size=size)
        tv.append(v)
        tc.append(c)
    return sv, sc, tv, tc


def rays(views) -> int:
    return sum(abi.rays_of(v) for v in views)


def find_surface_ray(ctx, fid, params, seed=5, radius=12.0, tries=64):
    """Seeded search for a ray that hits the fractal: a camera on a sphere of the
    given radius aimed near the origin, marched once with an FP64 DE and a 20-step
    bisection.  Returns (origin, unit direction, hit distance)."""
    import numpy as np

    from . import runtime

    rng = random.Random(seed)
    for _ in range(tries):
        z = rng.uniform(-1.0, 1.0)
        phi = rng.uniform(0.0, 2.0 * math.pi)
        s = math.sqrt(max(0.0, 1.0 - z * z))
        org = (radius * s * math.cos(phi), radius * s * math.sin(phi), radius * z)
        target = (rng.uniform(-0.3, 0.3), rng.uniform(-0.3, 0.3), rng.uniform(-0.3, 0.3))
        v = abi.make_view(fid, 1, 1, org, target=target, fov_y_deg=1e-6, params=params, max_steps=4096,
                          max_dist=4.0 * radius, eps_coef=1e-9, eps_floor=0.0, refine_budget=20)
        g = runtime.GBuffer.allocate(1)
        ctx.forward([v], g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=64))
        out = g.numpy()
        if out["normal"][0, 3] > 0.5:
            d = np.asarray(v.fwd, dtype=np.float64)
            return org, d / np.linalg.norm(d), float(out["depth64"][0])
    raise RuntimeError("no surface ray found")


def deepzoom_4096(resolve, ctx, size=4096, tiles=4, standoff=1e-5, fov_deg=0.01, seed=5):
    """Deep-zoom precision workload: Mandelbox scale -1.5, 30 iterations, a camera
    `standoff` from the surface along a searched ray, FOV 0.01 deg, a 4096^2 frame as
    tiles x tiles tiles; eps = 1e-8 t, FP64 ray origin/direction/t, bisection hit
    refinement (20 steps)."""
    fid = resolve(MANDELBOX)
    params = mandelbox_params(-1.5, 30)
    org, d, t = find_surface_ray(ctx, fid, params, seed=seed)
    cam = tuple(float(org[i] + d[i] * (t - standoff)) for i in range(3))
    target = tuple(float(cam[i] + d[i]) for i in range(3))
    views = []
    step = size // tiles
    for ty in range(tiles):
        for tx in range(tiles):
            views.append(abi.make_view(fid, size, size, cam, target=target, fov_y_deg=fov_deg, params=params,
                                       tile_x=tx * step, tile_y=ty * step, tile_w=step, tile_h=step,
                                       max_steps=512, max_dist=1.0, eps_coef=1e-8, eps_floor=0.0,
                                       refine_budget=20, normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=1e-8,
                                       flags=abi.ND_VIEW_DIR64))
    return views
