"""Parity of the 1080p Mandelbox configuration (Mandelbox scale -1.5, fold limit 1,
min radius^2 0.25, fixed radius^2 1, 15 iterations; 4 jittered rays per pixel from a
seed; at most 512 steps, eps 5e-5 t; one directional shadow ray per hit with
k = 16; box-shell orbit trap) on 128 x 96 crops of the frame, against the CPU
oracle on the same rays.

The jittered sample positions are part of the comparison: the kernel and the
oracle draw them from the same counter hash of (seed, the sample's place in the
frame), so every ray of the crop must be the same ray on both sides.  A depth that
agrees to 1e-4 across a pixel of this frame (1.6e-3 rad) would not survive a
different sample position on a slanted surface.  The same key makes a view cut
into tiles march the rays of the uncut view: a tiled call matches the whole one bit
for bit.

Tolerances.  This configuration's FP32 DE is far noisier than the others': 15
iterations of a scale -1.5 box fold amplify rounding along chaotic orbits, and the
normal's central difference uses h = eps(t) = 5e-5 t.  The reference's own FP32
arithmetic (the oracle run in FP32 on the same rays) misses the FP64 result by about
as much as the GPU does (measured on these crops: normal p99 about 13.9 and 5.7 degrees,
trap p99 0.042 and 0.019, 25 and 100 decisions flipped among the rays that are
stable under a 1e-4 DE perturbation).  So the GPU is held to the FP64 oracle with
that FP32 noise floor, measured in the test on the same rays: strict integer
mismatches at most 1.5x the FP32 oracle's plus 0.1 % + 2, normal p99 at most 1.5x its
p99 + 0.5 degree, trap p99 at most 1.5x + 1e-3; the hit fraction and mean step
count within 2 %; depth p99 relative error <= 1e-4 outright (the required depth bound).
Shadow visibility is compared with the FP32 oracle: more than 1e-3 apart on at most
1 % of the stable hits.  The FP64-DE mode must match the FP64 oracle to 1e-9 in depth
with at most 2 hit differences.
"""

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads
from tests.parity_util import compare, policy_check

pytestmark = pytest.mark.gpu


def crop(tile):
    v = workloads.mandelbox_1080p(runtime.find_formula)[0]
    v.tile_x, v.tile_y, v.tile_w, v.tile_h = tile[0], tile[1], 128, 96
    return v


def run(ctx, v, de_precision=32):
    n = abi.rays_of(v)
    g = runtime.GBuffer.allocate(n)
    ctx.forward([v], g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=de_precision))
    st = ctx.stats()
    return g.numpy(), st


# a crop across the silhouette (hits and misses) and one inside the fractal
TILES = [(384, 480), (896, 492)]


@pytest.mark.parametrize("tile", TILES)
def test_c2_crop_matches_the_oracle(ctx, tile):
    from oracle import pyoracle

    v = crop(tile)
    assert v.spp == 4 and v.max_steps == 512 and v.shadow == 1 and v.trap.shape == abi.ND_TRAP_BOX
    gp, st = run(ctx, v)
    n = abi.rays_of(v)
    assert st.rays == n and st.timeouts == 0
    assert st.de_evals == int(gp["evals"].astype(np.int64).sum()) + st.trap_evals

    # the four samples of a pixel are different rays (jitter on)
    npix = v.tile_w * v.tile_h
    d = gp["depth64"].reshape(4, npix)
    hit_all = (gp["normal"][:, 3].reshape(4, npix) > 0.5).all(0)
    same = (d[0] == d[1]) & (d[1] == d[2]) & (d[2] == d[3]) & hit_all
    assert same.sum() <= 0.01 * max(hit_all.sum(), 1), "samples of a pixel coincide: no jitter"

    unstable, r64 = pyoracle.unstable_rays(v, workloads.MANDELBOX)
    r32 = pyoracle.render(v, workloads.MANDELBOX, precision=32)
    pol = policy_check(gp, r64, unstable)
    strict = pol.pop("strict_mask")
    c64 = compare(gp, r64, mask=strict)
    # the noise floor: the reference's FP32 arithmetic (the oracle in FP32) on the same rays
    floor = policy_check(r32, r64, unstable)
    floor.pop("strict_mask")
    f64 = compare(r32, r64, mask=strict)
    print("policy:", pol)
    print("FP32 oracle policy:", floor)
    print("vs FP64 oracle (stable short rays):", c64)
    print("FP32 oracle vs FP64 oracle:", f64)
    assert pol["strict_mismatch"] <= 1.5 * floor["strict_mismatch"] + 0.001 * pol["strict_rays"] + 2, (pol, floor)
    assert abs(pol["hit_frac_gpu"] - pol["hit_frac_f64"]) <= 0.02
    assert abs(pol["mean_steps_gpu"] - pol["mean_steps_f64"]) <= 0.02 * max(pol["mean_steps_f64"], 1.0)
    assert c64["depth_rel_p99"] <= 1e-4
    assert c64["normal_deg_p99"] <= 1.5 * f64["normal_deg_p99"] + 0.5
    assert c64["trap_abs_p99"] <= 1.5 * f64["trap_abs_p99"] + 1e-3

    both = (gp["normal"][:, 3] > 0.5) & (r32["normal"][:, 3] > 0.5) & strict
    dv = np.abs(gp["shadow"][both] - r32["shadow"][both])
    print("shadow |diff| > 1e-3:", float((dv > 1e-3).mean()), "visible mean", float(gp["shadow"][both].mean()))
    assert (dv > 1e-3).mean() <= 0.01


@pytest.mark.parametrize("tile", TILES[:1])
def test_c2_crop_fp64_de_matches_the_fp64_oracle(ctx, tile):
    from oracle import pyoracle

    v = crop(tile)
    gp, _ = run(ctx, v, de_precision=64)
    r64 = pyoracle.render(v, workloads.MANDELBOX, precision=64)
    c = compare(gp, r64)
    print("FP64 DE vs FP64 oracle:", c)
    assert c["hit_mismatch"] <= 2
    assert c["depth_rel_p99"] <= 1e-9


def test_c2_tiles_march_the_rays_of_the_whole_crop(ctx):
    # both calls batched (several views in one persistent launch): the crop with a
    # small second view, and the crop's four tiles
    from numericdream_b200 import shard

    v = crop(TILES[0])
    extra = crop((0, 0))
    extra.tile_w, extra.tile_h = 8, 8
    n = abi.rays_of(v)
    g1 = runtime.GBuffer.allocate(n + abi.rays_of(extra))
    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT)
    ctx.forward([v, extra], g1, opts)
    tiles = shard.split_tiles(v, 2, 2)
    g2 = runtime.GBuffer.allocate(n)
    ctx.forward(tiles, g2, opts)
    a, b = g1.numpy(), g2.numpy()
    off = 0
    for t in tiles:
        m = abi.rays_of(t)
        ys, xs = slice(t.tile_y - v.tile_y, t.tile_y - v.tile_y + t.tile_h), slice(t.tile_x - v.tile_x,
                                                                                  t.tile_x - v.tile_x + t.tile_w)
        for k in ("depth64", "steps", "evals", "shadow", "trap"):
            whole = a[k][:n].reshape(v.spp, v.tile_h, v.tile_w)[:, ys, xs]
            part = b[k][off:off + m].reshape(t.spp, t.tile_h, t.tile_w)
            np.testing.assert_array_equal(part, whole, err_msg=k)
        off += m
