"""The `@image` formula (formulas/heightmap_primitive.wgsl) with an image, on the GPU,
against the CPU oracle given the same prepared texels: its DE at points (FP64 to
1e-9 relative, FP32 within FP32 noise), a forward march of a view of it under the
boundary-case policy with the depth bound of the other parity tests, and the same
formula with no image (the sampler reports size 0, as the reference does when no image
is loaded)."""

import numpy as np
import pytest

from numericdream_b200 import abi, runtime
from tests.parity_util import compare, policy_check

pytestmark = pytest.mark.gpu

NAME = "heightmap_primitive"


def _image(h=48, w=64):
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    hgt = 0.5 + 0.3 * np.sin(xx / w * 6.0) * np.cos(yy / h * 4.0) + 0.15 * (xx > w * 0.6)
    rgba = np.stack([hgt, 0.8 * hgt, 0.3 * np.ones_like(hgt), np.ones_like(hgt)], -1)
    return runtime.prepare_image(rgba), (w, h)


def _view(fid, texels_dev, wh, slope, size=48, pos=(0.9, 1.3, -1.6)):
    # Size 1, Height 0.3, Base 0.02, luminance weights, no invert
    v = abi.make_view(fid, size, size, pos, fov_y_deg=60.0, params=[1.0, 0.3, 0.02, 0.2126, 0.7152, 0.0722, 0.0, 0.0],
                      max_steps=256, eps_coef=1e-4, eps_floor=0.0, normal_mode=abi.ND_NORMAL_CENTRAL,
                      normal_h_coef=1e-4)
    if texels_dev is not None:
        v.image_texels = texels_dev.data_ptr()
        v.image_width, v.image_height = wh
        v.image_slope[:] = [float(x) for x in slope]
    return v


def test_image_formula_matches_the_oracle(ctx):
    import torch

    from oracle import pyoracle

    if NAME not in runtime.formula_names():
        pytest.skip("the image formula is not in this build")
    fid = runtime.find_formula(NAME)
    (texels, slope), wh = _image()
    dev = torch.from_numpy(texels.view(np.int32)).cuda()
    pyoracle.set_image(texels, wh[0], wh[1], slope)
    try:
        rng = np.random.default_rng(3)
        pts = np.column_stack([rng.uniform(-1.2, 1.2, 512), rng.uniform(-0.4, 0.6, 512), rng.uniform(-1.2, 1.2, 512)])
        v = _view(fid, dev, wh, slope)
        for prec, tol in ((64, 1e-9), (32, 1e-3)):
            d, _, _ = ctx.de_points(v, pts, prec)
            ref, _, _ = pyoracle.de(NAME, list(v.params), pts, precision=64)
            rel = np.abs(d - ref) / np.maximum(np.abs(ref), 1e-3)
            print(f"image formula DE fp{prec}: median rel {np.median(rel):.2e} max {rel.max():.2e}")
            assert (np.median(rel) if prec == 32 else rel.max()) <= tol
        # the sampled height reaches the DE: with the image the field differs from none
        d_none, _, _ = ctx.de_points(_view(fid, None, wh, slope), pts, 64)
        assert np.abs(d_none - d).max() > 1e-3

        n = abi.rays_of(v)
        g = runtime.GBuffer.allocate(n)
        ctx.forward([v], g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
        gp = g.numpy()
        unstable, r64 = pyoracle.unstable_rays(v, NAME)
        pol = policy_check(gp, r64, unstable)
        strict = pol.pop("strict_mask")
        c = compare(gp, r64, mask=strict)
        print("image formula march: policy", pol, "vs FP64 oracle", c)
        assert pol["ok"], pol
        assert c["hits_ref"] > 0.2 * n
        assert c["depth_rel_p99"] <= 1e-4
    finally:
        pyoracle.set_image(None)


def test_image_formula_without_an_image(ctx):
    from oracle import pyoracle

    if NAME not in runtime.formula_names():
        pytest.skip("the image formula is not in this build")
    fid = runtime.find_formula(NAME)
    v = _view(fid, None, (0, 0), [0, 0, 0, 0])
    rng = np.random.default_rng(4)
    pts = rng.uniform(-1.5, 1.5, (256, 3))
    d, _, _ = ctx.de_points(v, pts, 64)
    ref, _, _ = pyoracle.de(NAME, list(v.params), pts, precision=64)
    np.testing.assert_allclose(d, ref, rtol=1e-9, atol=1e-12)
