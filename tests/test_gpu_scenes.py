"""GPU parity of multi-instance scenes (nd_march_forward_scenes: scene_de,
template.wgsl:1756-1779 with combine_de, apply_carves and eval_mixed) against the CPU
oracle's scene path, with the tolerances of the single-instance parity tests:
boundary-case policy for hit/miss and step counts, depth p99 relative error vs FP64
<= 1e-4, normal p99 <= 2 degrees (3 for the discontinuous-gradient smooth mix),
trap p99 <= 1e-3 over stable short rays both runs hit.  Scenes use the formulas of
the default formula group (mandelbrot, amazingbox_box, menger3_ifs,
pseudokleinian_kleinian)."""

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads
from tests.parity_util import compare, policy_check

pytestmark = pytest.mark.gpu


def _fid(name):
    return runtime.find_formula(name)


def _view(size=64, cam=(0.0, 0.4, -3.2), **kw):
    kw.setdefault("max_steps", 256)
    return abi.make_view(_fid(workloads.MANDELBULB), size, size, cam, fov_y_deg=55.0, **kw)


def _forward(ctx, views, view_scene, scenes, de_precision=32):
    g = runtime.GBuffer.allocate(workloads.rays(views))
    ctx.forward_scenes(views, view_scene, scenes, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT,
                                                                      de_precision=de_precision))
    return g.numpy(), ctx.stats()


def _check(gpu, view, scene, normal_deg=2.0, min_hits=50):
    from oracle import pyoracle

    unstable, base = pyoracle.unstable_scene_rays(view, scene, runtime.formula_name)
    pol = policy_check(gpu, base, unstable)
    strict = pol.pop("strict_mask")
    print("policy:", pol)
    assert pol["ok"], pol
    c = compare(gpu, base, mask=strict)
    print("vs oracle f64 (stable short rays):", c)
    assert c["hits_ref"] >= min_hits
    if "depth_rel_p99" in c:
        assert c["depth_rel_p99"] <= 1e-4
        assert c["normal_deg_p99"] <= normal_deg
        assert c["trap_abs_p99"] <= 1e-3
    return c


def _slice(g, lo, hi):
    return {k: v[lo:hi] for k, v in g.items()}


def test_single_identity_instance_equals_the_plain_view(ctx):
    prm = workloads.mandelbulb_params(8.0, 10)
    v = _view(96, params=prm)
    inst = abi.make_instance(_fid(workloads.MANDELBULB), params=prm)
    inst.trap = v.trap
    g_plain = runtime.GBuffer.allocate(workloads.rays([v]))
    ctx.forward([v], g_plain, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    a = g_plain.numpy()
    b, st = _forward(ctx, [v], [0], [abi.make_scene([inst])])
    # the scene kernels are separate compilations of the same ray program: the
    # integer outputs agree ray for ray but for a few rounding-decided rays
    for k in ("steps", "evals"):
        assert (a[k] == b[k]).mean() >= 0.99, k
    both = (a["normal"][:, 3] > 0.5) & (b["normal"][:, 3] > 0.5)
    assert ((a["normal"][:, 3] > 0.5) == (b["normal"][:, 3] > 0.5)).mean() >= 0.995
    rel = np.abs(a["depth64"][both] - b["depth64"][both]) / a["depth64"][both]
    assert np.percentile(rel, 99) <= 1e-5
    assert st.rays == workloads.rays([v]) and st.timeouts == 0


def test_two_instances_smooth_union_and_carve(ctx):
    box = workloads.mandelbox_params(-1.5, 10)
    bulb = workloads.mandelbulb_params(8.0, 8)
    a = abi.make_instance(_fid(workloads.MANDELBOX), params=box, offset=(-0.9, 0.0, 0.0), scale=(0.3, 0.3, 0.3),
                          rotation_deg=(0.0, 30.0, 0.0))
    b = abi.make_instance(_fid(workloads.MANDELBULB), params=bulb, offset=(0.7, 0.0, 0.0), scale=(0.8, 0.8, 0.8),
                          combine_mode=abi.ND_COMBINE_SMOOTH_MIN, blend_k=0.15)
    scene = abi.make_scene([a, b], carves=[(0.7, 0.0, -0.7, 0.35), (-0.9, 0.5, -0.5, 0.25)])
    v = _view(96)
    g, st = _forward(ctx, [v], [0], [scene])
    _check(g, v, scene)
    assert st.timeouts == 0


@pytest.mark.parametrize("mode", [abi.ND_COMBINE_SMOOTH_MIN, abi.ND_COMBINE_SMOOTH_MAX, abi.ND_COMBINE_SMOOTH_INV_MAX,
                                  abi.ND_COMBINE_SMOOTH_MIN_LIN, abi.ND_COMBINE_SMOOTH_MIN_NLIN,
                                  abi.ND_COMBINE_SMOOTH_MIX])
def test_combine_modes(ctx, mode):
    bulb = workloads.mandelbulb_params(8.0, 8)
    menger = workloads.menger_params(4)
    a = abi.make_instance(_fid(workloads.MANDELBULB), params=bulb, offset=(0.0, 0.0, 0.0))
    b = abi.make_instance(_fid(workloads.MENGER), params=menger, offset=(0.35, 0.2, -0.3), scale=(0.7, 0.7, 0.7),
                          rotation_deg=(20.0, 35.0, 0.0), combine_mode=mode, blend_k=0.2)
    scene = abi.make_scene([a, b])
    v = _view(80)
    g, _ = _forward(ctx, [v], [0], [scene])
    _check(g, v, scene, normal_deg=3.0 if mode == abi.ND_COMBINE_SMOOTH_MIX else 2.0,
           min_hits=0 if mode == abi.ND_COMBINE_SMOOTH_MAX else 50)


def test_hybrid_mixins(ctx):
    box = workloads.mandelbox_params(-1.5, 10)
    bulb = workloads.mandelbulb_params(8.0, 8)
    inst = abi.make_instance(_fid(workloads.MANDELBOX), params=box, scale=(0.5, 0.5, 0.5),
                             mixins=[(_fid(workloads.MANDELBULB), 1, bulb)], hybrid_base_iters=2,
                             hybrid_total_iters=10)
    scene = abi.make_scene([inst])
    v = _view(96)
    g, _ = _forward(ctx, [v], [0], [scene])
    _check(g, v, scene)


def test_hidden_instances_and_mixed_batch(ctx):
    """Scene views and single-instance views in one batched call; a hidden instance
    contributes nothing."""
    bulb = workloads.mandelbulb_params(8.0, 8)
    kl = workloads.pseudo_kleinian_params(1.0)
    a = abi.make_instance(_fid(workloads.MANDELBULB), params=bulb, scale=(0.9, 0.9, 0.9))
    hidden = abi.make_instance(_fid(workloads.PSEUDO_KLEINIAN), params=kl, offset=(0.0, 0.0, -1.0), hidden=True)
    s_vis = abi.make_scene([a])
    s_hid = abi.make_scene([a, hidden])
    v_plain = abi.make_view(_fid(workloads.MANDELBOX), 48, 48, (0.0, 0.0, -4.5), fov_y_deg=60.0,
                            params=workloads.mandelbox_params(-1.5, 10), max_steps=256)
    v1, v2 = _view(64), _view(64)
    views = [v1, v_plain, v2]
    g, st = _forward(ctx, views, [0, -1, 1], [s_vis, s_hid])
    n1, n2 = workloads.rays([v1]), workloads.rays([v_plain])
    g1, gp, g2 = _slice(g, 0, n1), _slice(g, n1, n1 + n2), _slice(g, n1 + n2, n1 + n2 + n1)
    for k in ("depth64", "steps", "evals", "trap"):
        np.testing.assert_array_equal(g1[k], g2[k], err_msg=k)
    _check(g1, v1, s_vis)
    from oracle import pyoracle

    unstable, base = pyoracle.unstable_rays(v_plain, workloads.MANDELBOX)
    pol = policy_check(gp, base, unstable)
    pol.pop("strict_mask")
    assert pol["ok"], pol
    assert st.rays == workloads.rays(views)


def test_formulas_outside_one_set_are_refused(ctx):
    """Scenes need every formula of the call in one compiled formula group."""
    outside = None
    for name in runtime.formula_names():
        if name not in (workloads.MANDELBULB, workloads.MANDELBOX, workloads.MENGER, workloads.PSEUDO_KLEINIAN):
            outside = name
            break
    assert outside is not None
    a = abi.make_instance(_fid(workloads.MANDELBULB), params=workloads.mandelbulb_params(8.0, 8))
    b = abi.make_instance(_fid(outside), params=[0.5])
    v = _view(16)
    g = runtime.GBuffer.allocate(workloads.rays([v]))
    with pytest.raises(runtime.NDError) as e:
        ctx.forward_scenes([v], [0], [abi.make_scene([a, b])], g)
    assert e.value.status == abi.ND_ERR_UNSUPPORTED


def test_graph_replay_of_a_scene_call(ctx):
    """nd_graph_capture_scenes: a replay writes what the direct scene call wrote, and
    keeps marching the captured scenes after the caller's tables change."""
    import torch

    box = workloads.mandelbox_params(-1.5, 10)
    bulb = workloads.mandelbulb_params(8.0, 8)
    a = abi.make_instance(_fid(workloads.MANDELBOX), params=box, offset=(-0.9, 0.0, 0.0), scale=(0.3, 0.3, 0.3))
    b = abi.make_instance(_fid(workloads.MANDELBULB), params=bulb, offset=(0.7, 0.0, 0.0), scale=(0.8, 0.8, 0.8),
                          combine_mode=abi.ND_COMBINE_SMOOTH_MIN, blend_k=0.15)
    scenes = [abi.make_scene([a, b], carves=[(0.7, 0.0, -0.7, 0.35)])]
    v_plain = abi.make_view(_fid(workloads.MANDELBOX), 48, 48, (0.0, 0.0, -4.5), fov_y_deg=60.0,
                            params=box, max_steps=256)
    views = [_view(64), v_plain]
    view_scene = [0, -1]
    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT)
    g1, _ = _forward(ctx, views, view_scene, scenes)
    gb = runtime.GBuffer.allocate(workloads.rays(views))
    graph = ctx.capture_scenes(views, view_scene, scenes, gb, opts)
    try:
        # the caller's scene table changes after the capture; the graph keeps its copy
        scenes[0].instances[0].offset[0] = 5.0
        for _ in range(2):
            graph.launch()
            torch.cuda.synchronize()
            g2 = gb.numpy()
            for k in ("depth64", "steps", "evals", "trap", "normal"):
                np.testing.assert_array_equal(g1[k], g2[k], err_msg=k)
        assert ctx.stats().rays == workloads.rays(views)
    finally:
        graph.close()
    with pytest.raises(runtime.NDError) as e:
        ctx.capture_scenes(views, [0, 1], scenes, gb, opts)
    assert e.value.status == abi.ND_ERR_INVALID
