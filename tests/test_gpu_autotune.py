"""The autotuner (nd_autotune) and its cache on disk (nd_tune_cache_save / _load).

The launch configuration must not change any ray's result: the persistent march at
64, 128 and 256 threads per block and at several residencies gives the same bits.
The tuner's pick is a configuration that fits on the SM (every block of the
persistent grid resident), later forwards of the same formula set use it, and the
cache written to disk reads back as the same entries."""

import json

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu

MAX_THREADS_PER_SM = 2048


def _views():
    return workloads.batched_64(runtime.find_formula, nviews=8, min_side=48, max_side=160, seed=21)


def test_block_sizes_and_residency_give_the_same_rays(ctx):
    views = _views()
    n = workloads.rays(views)
    ref = None
    for block in (64, 128, 256):
        for per_sm in (0, -2, 3):
            g = runtime.GBuffer.allocate(n)
            ctx.forward(views, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, block=block,
                                                    blocks_per_sm=per_sm, refill_threshold=4))
            st = ctx.stats()
            assert st.rays == n
            out = g.numpy()
            if ref is None:
                ref = out
                continue
            for k in ("depth64", "steps", "evals", "normal", "trap", "iters", "shade"):
                np.testing.assert_array_equal(out[k], ref[k], err_msg=f"block {block}, blocks/SM {per_sm}: {k}")
    with pytest.raises(runtime.NDError):
        ctx.forward(views, runtime.GBuffer.allocate(n), runtime.make_opts(block=96))


def test_autotune_picks_a_resident_configuration_and_caches_it(ctx, tmp_path):
    views = _views()
    n = workloads.rays(views)
    g = runtime.GBuffer.allocate(n)
    r = ctx.autotune(views, g)
    print("tuned:", r.kernel, r.block, r.blocks_per_sm, r.refill_threshold, f"{r.rays_per_s / 1e6:.0f} Mrays/s")
    assert r.kernel in (abi.ND_KERNEL_PLAIN, abi.ND_KERNEL_PERSISTENT)
    assert r.rays_per_s > 0
    if r.kernel == abi.ND_KERNEL_PERSISTENT:
        assert r.block in (64, 128, 256)
        assert 1 <= r.blocks_per_sm and r.blocks_per_sm * r.block <= MAX_THREADS_PER_SM
        assert 3 <= r.refill_threshold <= 12
    # later forwards with default options run the pick
    ctx.forward(views, g, runtime.make_opts())
    assert ctx.stats().kernel == r.kernel
    # the cache: saved, then read back as the same entries
    path = str(tmp_path / "tune.json")
    runtime.Context.tune_cache_save(path)
    entries = json.load(open(path))
    mine = [e for e in entries if "group:mixed4" in e["key"]]
    assert mine, entries
    e = mine[0]
    assert e["kernel"] == r.kernel and e["refill_threshold"] == r.refill_threshold
    if r.kernel == abi.ND_KERNEL_PERSISTENT:
        assert e["block"] == r.block
    import torch

    assert torch.cuda.get_device_name(0) in e["key"]
    # the winner is the FP32 DE's: an FP64-DE forward of the same formulas, whose
    # kernels fit fewer blocks per SM, keeps the defaults
    assert e["key"].endswith("|fp32")
    assert not any(x["key"].endswith("|fp64") for x in entries)
    assert runtime.Context.tune_cache_load(path) == len(entries)
    with pytest.raises(runtime.NDError) as err:
        runtime.Context.tune_cache_load(str(tmp_path / "missing.json"))
    assert err.value.status == abi.ND_ERR_NOT_FOUND


def test_untuned_single_small_view_runs_the_plain_launch():
    """With no tuning entry, one view with no more rays than the persistent grid has
    threads runs the plain launch (one ray per thread, nothing to refill) with the plain
    launch's results; several views run the persistent march."""
    c = runtime.Context(0)
    try:
        small = workloads.mandelbulb_256(runtime.find_formula)
        n = workloads.rays(small)
        g = runtime.GBuffer.allocate(n)
        c.forward(small, g, runtime.make_opts())
        assert c.stats().kernel == abi.ND_KERNEL_PLAIN
        auto = g.numpy()
        c.forward(small, g, runtime.make_opts(kernel=abi.ND_KERNEL_PLAIN))
        plain = g.numpy()
        for k in ("depth64", "steps", "evals", "normal", "trap", "shade"):
            np.testing.assert_array_equal(auto[k], plain[k], err_msg=k)
        views = _views()
        c.forward(views, runtime.GBuffer.allocate(workloads.rays(views)), runtime.make_opts())
        assert c.stats().kernel == abi.ND_KERNEL_PERSISTENT
        # one view with more rays than the grid has threads: the persistent march
        big = workloads.mandelbox_1080p(runtime.find_formula)
        assert len(big) == 1
        c.forward(big, runtime.GBuffer.allocate(workloads.rays(big)), runtime.make_opts())
        assert c.stats().kernel == abi.ND_KERNEL_PERSISTENT
    finally:
        c.close()
