"""GPU parity of the empty-space accelerator: the grid build (cs_build_accel,
template.wgsl:5412-5431) against the CPU oracle's grid, and the accelerated march
(accel_skip in march_to :1890-1900 and visibility_march :2297-2303) against the
oracle's accelerated march, with the single-view parity tolerances (boundary-case
policy for hit/miss and steps; depth p99 <= 1e-4, normal p99 <= 2 degrees, trap p99
<= 1e-3 over stable short rays both hit)."""

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads
from tests.parity_util import compare, policy_check

pytestmark = pytest.mark.gpu


def _fid(name):
    return runtime.find_formula(name)


def _forward(ctx, views, kernel=abi.ND_KERNEL_PERSISTENT, de_precision=32):
    g = runtime.GBuffer.allocate(workloads.rays(views))
    ctx.forward(views, g, runtime.make_opts(kernel=kernel, de_precision=de_precision))
    return g.numpy(), ctx.stats()


def _check(gpu, view, name):
    from oracle import pyoracle

    unstable, base = pyoracle.unstable_rays(view, name)
    pol = policy_check(gpu, base, unstable)
    strict = pol.pop("strict_mask")
    print("policy:", pol)
    assert pol["ok"], pol
    c = compare(gpu, base, mask=strict)
    print("vs oracle f64 (stable short rays):", c)
    assert c["hits_ref"] >= 50
    assert c["depth_rel_p99"] <= 1e-4
    assert c["normal_deg_p99"] <= 2.0
    assert c["trap_abs_p99"] <= 1e-3
    return c


def _mandelbox_view(size=96, **kw):
    return abi.make_view(_fid(workloads.MANDELBOX), size, size, (0.3, 0.6, -4.2), fov_y_deg=60.0,
                         params=workloads.mandelbox_params(-1.5, 10), max_steps=256, **kw)


@pytest.mark.parametrize("precision", [32, 64])
def test_grid_matches_the_oracle(ctx, precision):
    from oracle import pyoracle

    v = _mandelbox_view(accel_res=32, accel_levels=5, accel_safety=0.92)
    grid, prm = ctx.accel_grid(v, precision)
    want, prm_o = pyoracle.accel_grid(v, workloads.MANDELBOX, 64)
    np.testing.assert_array_equal(prm, prm_o)
    err = np.abs(grid.astype(np.float64) - want.astype(np.float64))
    print("grid |err| max", err.max(), "cells", grid.size, "nonzero", int((want > 0).sum()))
    assert (want > 0).sum() > 0.3 * want.size
    # FP32 fast-math DE: relative 1e-3 of the distance; FP64 DE: f32 rounding
    tol = (1e-3 if precision == 32 else 1e-6) * np.abs(want) + 1e-5
    assert (err <= tol).mean() >= 0.999
    assert err.max() <= 0.05


@pytest.mark.parametrize("name", [workloads.MANDELBULB, workloads.MANDELBOX, workloads.MENGER])
def test_accelerated_march_parity(ctx, name):
    params = {workloads.MANDELBULB: workloads.mandelbulb_params(8.0, 10),
              workloads.MANDELBOX: workloads.mandelbox_params(-1.5, 10),
              workloads.MENGER: workloads.menger_params(4)}[name]
    cam = (0.5, 0.9, -2.6) if name != workloads.MANDELBOX else (0.3, 0.6, -4.2)
    v = abi.make_view(_fid(name), 96, 96, cam, fov_y_deg=60.0, params=params, max_steps=256, accel_res=48,
                      accel_levels=6, accel_safety=0.92)
    g, st = _forward(ctx, [v])
    assert st.accel_voxels == 6 * 48 ** 3 and st.accel_ms > 0 and st.timeouts == 0
    _check(g, v, name)
    # against the same view without the accelerator: the same surface, fewer evaluations
    v0 = abi.nd_view_desc.from_buffer_copy(v)
    v0.accel_res = 0
    g0, st0 = _forward(ctx, [v0])
    h, h0 = g["normal"][:, 3] > 0.5, g0["normal"][:, 3] > 0.5
    print("hits", h.sum(), h0.sum(), "march evals", st.march_evals, st0.march_evals)
    assert (h != h0).mean() <= 0.01
    assert st.march_evals < st0.march_evals
    assert st0.accel_voxels == 0


def test_shadows_scenes_and_fp64_with_the_accelerator(ctx):
    from oracle import pyoracle

    # shadow rays take the jumps too
    v = _mandelbox_view(80, shadow=1, light_dir=(0.4, 0.8, -0.45), accel_res=32, accel_levels=5)
    g, _ = _forward(ctx, [v])
    _check(g, v, workloads.MANDELBOX)
    unstable, base = pyoracle.unstable_rays(v, workloads.MANDELBOX)
    both = (g["normal"][:, 3] > 0.5) & (base["normal"][:, 3] > 0.5) & ~unstable
    assert (np.abs(g["shadow"][both] - base["shadow"][both]) > 1e-3).mean() <= 0.02
    # FP64 DE
    g64, _ = _forward(ctx, [v], de_precision=64)
    c = compare(g64, base)
    assert c["hit_mismatch"] <= 0.002 * c["rays"] + 2 and c["depth_rel_p99"] <= 1e-6
    # a scene view
    bulb = workloads.mandelbulb_params(8.0, 8)
    a = abi.make_instance(_fid(workloads.MANDELBULB), params=bulb, offset=(-0.6, 0.0, 0.0), scale=(0.6,) * 3)
    b = abi.make_instance(_fid(workloads.MANDELBOX), params=workloads.mandelbox_params(-1.5, 10),
                          offset=(0.7, 0.0, 0.0), scale=(0.25,) * 3, combine_mode=abi.ND_COMBINE_SMOOTH_MIN,
                          blend_k=0.1)
    scene = abi.make_scene([a, b])
    vs = abi.make_view(_fid(workloads.MANDELBULB), 80, 80, (0.0, 0.4, -3.0), fov_y_deg=55.0, max_steps=256,
                       accel_res=32, accel_levels=5)
    gs = runtime.GBuffer.allocate(workloads.rays([vs]))
    ctx.forward_scenes([vs], [0], [scene], gs, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    gs = gs.numpy()
    unstable, base = pyoracle.unstable_scene_rays(vs, scene, runtime.formula_name)
    pol = policy_check(gs, base, unstable)
    pol.pop("strict_mask")
    assert pol["ok"], pol


def test_batched_views_with_and_without_the_accelerator(ctx):
    views = workloads.batched_64(_fid, nviews=8, max_side=160)
    for i, v in enumerate(views):
        if i % 2 == 0:
            v.accel_res, v.accel_levels, v.accel_safety = 32, 6, 0.92
    g, st = _forward(ctx, views)
    assert st.accel_voxels == 4 * 6 * 32 ** 3
    off = 0
    for i, v in enumerate(views):
        n = workloads.rays([v])
        gi = {k: a[off:off + n] for k, a in g.items()}
        single, _ = _forward(ctx, [v])
        # the batched accelerated march (the formula group's kernel) against the
        # single-view one (the formula's own kernel): separate compilations of the
        # FP32 DE round differently in the last bits, so rays agree but for a few
        h, hs = gi["normal"][:, 3] > 0.5, single["normal"][:, 3] > 0.5
        assert (h == hs).mean() >= 0.99, i
        assert (gi["steps"] == single["steps"]).mean() >= 0.97, i
        both = h & hs
        if both.any():
            rel = np.abs(gi["depth64"][both] - single["depth64"][both]) / single["depth64"][both]
            assert np.percentile(rel, 99) <= 1e-4, i
        off += n


def test_graph_replay_with_the_accelerator(ctx):
    v = _mandelbox_view(64, accel_res=32, accel_levels=4)
    g1, _ = _forward(ctx, [v])
    import torch

    gb = runtime.GBuffer.allocate(workloads.rays([v]))
    graph = ctx.capture([v], gb, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    try:
        graph.launch()
        torch.cuda.synchronize()
        g2 = gb.numpy()
    finally:
        graph.close()
    for k in ("depth64", "steps", "evals"):
        np.testing.assert_array_equal(g1[k], g2[k], err_msg=k)


def test_accelerator_refusals(ctx):
    v = _mandelbox_view(16, accel_res=32)
    g = runtime.GBuffer.allocate(workloads.rays([v]))
    with pytest.raises(runtime.NDError) as e:
        ctx.forward([v], g, runtime.make_opts(kernel=abi.ND_KERNEL_PLAIN))
    assert e.value.status == abi.ND_ERR_UNSUPPORTED
    bad = abi.nd_view_desc.from_buffer_copy(v)
    bad.accel_safety = 1.5
    with pytest.raises(runtime.NDError) as e:
        ctx.forward([bad], g)
    assert e.value.status == abi.ND_ERR_INVALID
    # FP32 DE with FP64 (deep-zoom) ray directions
    dz = abi.nd_view_desc.from_buffer_copy(v)
    dz.flags = abi.ND_VIEW_DIR64
    with pytest.raises(runtime.NDError) as e:
        ctx.forward([dz], g)
    assert e.value.status == abi.ND_ERR_UNSUPPORTED
    # the allocation-free entry has no grid memory (refused before it sets anything up)
    import ctypes as C

    fn = runtime.load_library().nd_march_forward_noalloc
    fn.restype = C.c_int32
    fn.argtypes = [C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(abi.nd_march_opts),
                   C.POINTER(abi.nd_gbuffer), C.c_void_p]
    g.trap = None
    g.iters = None
    gb = g.as_abi()
    assert fn((abi.nd_view_desc * 1)(v), 1, None, C.byref(gb), None) == abi.ND_ERR_UNSUPPORTED
