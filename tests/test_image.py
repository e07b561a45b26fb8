"""Formula images: nd_image_prepare against an independent numpy restatement of the
reference's preparation of a height map (src/gpu/height_maps.zig:264-320: 16-bit
quantisation, per-texel slope from the 2 x 2 block, block-maxima dilation over 8 + 2 and
64 + 2 texels, slope codes ceil(16 (log2(1.001 s) - 1) + 255) in 1..255), and the translator
taking the `@image` formula.  Runs without a GPU."""

import numpy as np
import pytest

from numericdream_b200 import runtime


def _round(x):
    # the reference's @round: halves away from zero (np.round goes to even)
    f = np.floor(x)
    return np.where(x - f >= np.float32(0.5), f + np.float32(1.0), f).astype(np.float32)


def reference_prepare(rgba):
    a = np.clip(rgba.astype(np.float32), 0.0, 1.0)
    v = (_round(a * np.float32(65535.0)) / np.float32(65535.0)).astype(np.float32)
    h, w = v.shape[:2]
    x1 = np.minimum(np.arange(w) + 1, w - 1)
    y1 = np.minimum(np.arange(h) + 1, h - 1)
    a_, b_ = v, v[:, x1]
    c_, d_ = v[y1, :], v[y1][:, x1]
    dx = np.maximum(np.abs(b_ - a_), np.abs(d_ - c_))
    dy = np.maximum(np.abs(c_ - a_), np.abs(d_ - b_))
    g = np.sqrt(dx * dx + dy * dy).astype(np.float32)
    glob = g.reshape(-1, 4).max(0)

    def dilate_line(x, r):
        # block maxima forward and backward within blocks of 2 r + 1 samples; a window
        # [j - r, j + r] (clamped at the ends) takes the backward maximum at its start
        # and the forward maximum at its end, as the reference computes it (near the
        # ends this can reach past the clamped window, within the start's block)
        n, k = x.shape[0], 2 * r + 1
        fwd, bwd = x.copy(), x.copy()
        for i in range(1, n):
            if i % k:
                fwd[i] = np.maximum(fwd[i - 1], x[i])
        for i in range(n - 2, -1, -1):
            if (i + 1) % k:
                bwd[i] = np.maximum(bwd[i + 1], x[i])
        j = np.arange(n)
        return np.maximum(bwd[np.maximum(j - r, 0)], fwd[np.minimum(j + r, n - 1)])

    def dilate(x, r):
        rows = np.stack([dilate_line(x[i], r) for i in range(h)])
        return np.stack([dilate_line(rows[:, jj], r) for jj in range(w)], 1)

    near, far = dilate(g, 10), dilate(g, 66)

    def code(s):
        with np.errstate(divide="ignore"):
            steps = np.ceil(np.float32(16.0) * (np.log2(s * np.float32(1.001)) - np.float32(1.0)) + np.float32(255.0))
        return np.where(s > 0, np.clip(steps, 1, 255), 0).astype(np.uint32)

    def pack(s):
        c = code(s.reshape(-1, 4))
        return c[:, 0] | (c[:, 1] << 8) | (c[:, 2] << 16) | (c[:, 3] << 24)

    q = _round(v.reshape(-1, 4) * np.float32(65535.0)).astype(np.uint32)
    t = np.zeros((h * w, 4), dtype=np.uint32)
    t[:, 0] = q[:, 0] | (q[:, 1] << 16)
    t[:, 1] = q[:, 2] | (q[:, 3] << 16)
    t[:, 2] = pack(near)
    t[:, 3] = pack(far)
    return t, (glob * np.float32(1.001)).astype(np.float32)


def _codes(word):
    return np.stack([(word >> (8 * k)) & 0xFF for k in range(4)], -1).astype(np.int64)


@pytest.mark.parametrize("shape", [(1, 1), (7, 5), (40, 61), (150, 3)])
def test_prepare_matches_the_reference_algorithm(ndlib, shape):
    rng = np.random.default_rng(sum(shape))
    h, w = shape
    # a smooth field plus noise and a hard edge, alpha premultiplied into RGB
    yy, xx = np.mgrid[0:h, 0:w]
    base = 0.5 + 0.4 * np.sin(xx * 0.3) * np.cos(yy * 0.2)
    rgba = np.stack([base, base * 0.5, (xx > w // 2).astype(float), np.ones_like(base)], -1)
    rgba[..., :3] += rng.normal(0.0, 0.02, (h, w, 3))
    rgba[..., 3] = rng.uniform(0.5, 1.0, (h, w))
    rgba[..., :3] *= rgba[..., 3:4]
    t, s = runtime.prepare_image(rgba)
    rt, rs = reference_prepare(rgba)
    t = t.reshape(-1, 4)
    np.testing.assert_array_equal(t[:, :2], rt[:, :2])  # the 16-bit channel values
    np.testing.assert_allclose(s, rs, rtol=1e-6)
    for col in (2, 3):  # slope codes: equal but where log2 rounds across an integer step
        diff = np.abs(_codes(t[:, col]) - _codes(rt[:, col]))
        assert diff.max() <= 1 and (diff > 0).mean() <= 0.01


def test_prepare_rejects_bad_sizes(ndlib):
    with pytest.raises(runtime.NDError):
        runtime.prepare_image(np.zeros((2049, 1, 4), np.float32))


def test_the_image_formula_translates():
    from numericdream_b200 import build
    from numericdream_b200.translator import translate

    if not build.reference_root():
        pytest.skip("the reference's formula files are not here")
    path, src = build.formula_sources()["heightmap_primitive"]
    tf = translate(src, "heightmap_primitive")
    assert "ndw::image_info<T>(p)" in tf.cpp and "ndw::image_sample<T>" in tf.cpp
    assert "image" in tf.features
