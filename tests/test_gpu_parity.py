"""GPU parity of the sphere-tracing kernels against the CPU oracle (through the C ABI).

Tolerances (FP32 DE on the GPU against the FP64 oracle on the same rays):
* hit/miss and probe-step counts follow the boundary-case policy of
  tests/parity_util.py: rays that are stable under a 1e-4 relative perturbation of
  every DE value and end within 64 probe steps must agree ray for ray (at most
  0.1% + 1 may differ); over all rays the hit fraction and the mean step count
  must agree within 2%;
* depth: p99 relative error vs FP64 <= 1e-4 over stable short rays both runs hit;
* normals: p99 angle vs FP64 <= 2 degrees (the default build's FP32 DE uses the
  GPU's fast sin/cos/pow approximations, whose noise the central-difference
  normal amplifies by 1/h; a build with ND_ACCURATE_MATH=1 stays under 1 degree);
* trap p99 abs <= 1e-3.
For a single view the plain and persistent kernels run the same ray program with the
same view record and must agree bit for bit.
"""

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads
from tests.parity_util import compare, policy_check

pytestmark = pytest.mark.gpu

NORMAL_DEG_P99 = 2.0


def _run(ctx, views, kernel, de_precision=32, threshold=0):
    n = workloads.rays(views)
    g = runtime.GBuffer.allocate(n)
    ctx.forward(views, g, runtime.make_opts(kernel=kernel, de_precision=de_precision, refill_threshold=threshold))
    st = ctx.stats()
    return g.numpy(), st


def _oracle(views, precision):
    from oracle import pyoracle

    outs = []
    for v in views:
        outs.append(pyoracle.render(v, runtime.formula_name(v.formula), precision=precision))
    return {k: np.concatenate([o[k] for o in outs]) for k in outs[0]}


def _resolve(name):
    return runtime.find_formula(name)


def test_c1_small_parity(ctx):
    views = workloads.mandelbulb_256(_resolve, size=96)
    gp, st = _run(ctx, views, abi.ND_KERNEL_PERSISTENT)
    gl, _ = _run(ctx, views, abi.ND_KERNEL_PLAIN)
    for k in ("depth", "normal", "trap", "steps", "iters", "evals", "depth64"):
        np.testing.assert_array_equal(gp[k], gl[k], err_msg=f"plain vs persistent differ in {k}")
    r32 = _oracle(views, 32)
    r64 = _oracle(views, 64)
    c32 = compare(gp, r32)
    c64 = compare(gp, r64)
    print("vs oracle f32:", c32)
    print("vs oracle f64:", c64)
    n = c32["rays"]
    assert st.rays == n and st.timeouts == 0
    assert st.de_evals == int(gp["evals"].astype(np.int64).sum()) + st.trap_evals
    assert st.trap_evals == st.hits
    from oracle import pyoracle

    unstable, base = pyoracle.unstable_rays(views[0], "mandelbrot")
    pol = policy_check(gp, base, unstable)
    strict = pol.pop("strict_mask")
    print("policy:", pol)
    assert pol["ok"], pol
    c64 = compare(gp, r64, mask=strict)
    print("vs oracle f64 (stable short rays):", c64)
    assert c64["depth_rel_p99"] <= 1e-4
    assert c64["normal_deg_p99"] <= NORMAL_DEG_P99
    assert c64["trap_abs_p99"] <= 1e-3


@pytest.mark.parametrize("name", [workloads.MANDELBOX, workloads.MENGER, workloads.PSEUDO_KLEINIAN])
def test_formula_parity(ctx, name):
    fid = runtime.find_formula(name)
    params = {workloads.MANDELBOX: workloads.mandelbox_params(-1.5, 12),
              workloads.MENGER: workloads.menger_params(4),
              workloads.PSEUDO_KLEINIAN: workloads.pseudo_kleinian_params(1.0)}[name]
    v = abi.make_view(fid, 80, 64, (2.2, 1.3, -3.1), fov_y_deg=60.0, params=params, max_steps=256,
                      normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=1e-4, shadow=1,
                      light_dir=list(workloads.LIGHT_DIR), trap={"shape": abi.ND_TRAP_BOX})
    gp, st = _run(ctx, [v], abi.ND_KERNEL_PERSISTENT)
    from oracle import pyoracle

    r32 = _oracle([v], 32)
    unstable, r64 = pyoracle.unstable_rays(v, name)
    pol = policy_check(gp, r64, unstable)
    strict = pol.pop("strict_mask")
    c64 = compare(gp, r64, mask=strict)
    print(name, "policy:", pol, "f64 (stable short rays):", c64)
    assert pol["ok"], pol
    if c64["hits_ref"]:
        assert c64["depth_rel_p99"] <= 1e-4
        assert c64["normal_deg_p99"] <= NORMAL_DEG_P99
    both = (gp["normal"][:, 3] > 0.5) & (r32["normal"][:, 3] > 0.5) & strict
    sh_g = gp["shadow"][both]
    sh_r = r32["shadow"][both]
    if sh_g.size:
        # shadow rays are marches of their own (up to 40 steps); through the
        # pseudo-Kleinian lattice they are as rounding-sensitive as its primary
        # rays, so there only the mean visibility is compared
        if name == workloads.PSEUDO_KLEINIAN:
            assert abs(float(sh_g.mean()) - float(sh_r.mean())) <= 0.02
        else:
            assert np.mean(np.abs(sh_g - sh_r) > 1e-3) <= 0.01


def test_batched_mixed_parity(ctx):
    """Mixed formulas in one persistent launch and as plain per-view launches; both
    are checked view by view against the FP64 oracle under the policy."""
    views = workloads.batched_64(_resolve, nviews=8, min_side=24, max_side=64, seed=3)
    gp, st = _run(ctx, views, abi.ND_KERNEL_PERSISTENT)
    gl, _ = _run(ctx, views, abi.ND_KERNEL_PLAIN)
    from oracle import pyoracle

    assert st.rays == workloads.rays(views)
    off = 0
    for v in views:
        n = v.spp * v.tile_w * v.tile_h
        name = runtime.formula_name(v.formula)
        unstable, base = pyoracle.unstable_rays(v, name)
        for label, g in (("persistent", gp), ("plain", gl)):
            part = {k: g[k][off:off + n] for k in g}
            pol = policy_check(part, base, unstable, agg_tol=0.05)
            pol.pop("strict_mask")
            print(label, name, pol)
            assert pol["ok"], (label, name, pol)
        diff = int((gp["depth"][off:off + n] != gl["depth"][off:off + n]).sum())
        print("  plain vs persistent depth differences:", diff, "of", n)
        off += n


def test_fp64_de_mode(ctx):
    views = workloads.mandelbulb_256(_resolve, size=48)
    gp, _ = _run(ctx, views, abi.ND_KERNEL_PERSISTENT, de_precision=64)
    r64 = _oracle(views, 64)
    c = compare(gp, r64)
    print("fp64 DE:", c)
    assert c["hit_mismatch"] <= 2
    assert c["depth_rel_p99"] <= 1e-9
