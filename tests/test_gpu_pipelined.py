"""Forward calls enqueued back to back without waiting, as a renderer streams frames.

A forward call returns once its work is enqueued.  Its view table goes up on a side
stream into one of two device halves that calls alternate, and its host staging is
one of two pinned halves, so a call may be made while the previous one still marches.
Every frame of such a stream of calls must equal the same frame marched on its own:
different view sets call after call (so a half holding the wrong table would show),
on one stream and on two streams taken in turn."""

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu

KEYS = ("depth64", "steps", "evals", "normal", "trap", "shade")


def _frames():
    out = []
    for seed in (3, 4, 5, 6, 7):
        out.append(workloads.batched_64(runtime.find_formula, nviews=5 + seed, min_side=32, max_side=96, seed=seed))
    return out


def test_frames_enqueued_back_to_back_match_frames_marched_alone(ctx):
    import torch

    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, refill_threshold=4)
    frames = _frames()
    alone = []
    for views in frames:
        g = runtime.GBuffer.allocate(workloads.rays(views))
        ctx.forward(views, g, opts)
        torch.cuda.synchronize()
        alone.append(g.numpy())
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for nstreams in (1, 2):
        bufs = [runtime.GBuffer.allocate(workloads.rays(v)) for v in frames]
        for i, views in enumerate(frames * 2):  # ten calls, nothing waited for in between
            s = streams[i % nstreams]
            ctx.forward(views, bufs[i % len(frames)], opts, stream=s.cuda_stream)
        torch.cuda.synchronize()
        for i, want in enumerate(alone):
            got = bufs[i].numpy()
            for k in KEYS:
                np.testing.assert_array_equal(got[k], want[k], err_msg=f"{nstreams} stream(s), frame {i}: {k}")


def test_lite_shading_between_forward_calls(ctx):
    # forward, lite shading of it, then the next frame's forward, nothing waited for:
    # the lite call's view table goes up from the staging half the forward after next
    # reuses, so each lite image must equal the one made with everything synchronised
    import torch

    stops = [((0.05, 0.05, 0.22), 0.0, 0.2, 1.3), ((1.0, 0.95, 0.82), 1.0, 0.8, 1.7)]
    lights = [(abi.ND_LIGHT_GLOBAL, (0.4, 0.8, -0.45), (1.0, 0.95, 0.9), 1.2)]
    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT)
    frames = _frames()
    lites = [[abi.make_lite(stops, lights) for _ in v] for v in frames]
    want = []
    for views, lt in zip(frames, lites):
        g = runtime.GBuffer.allocate(workloads.rays(views))
        ctx.forward(views, g, opts)
        want.append(ctx.shade_lite(views, lt, g).cpu().numpy())
        torch.cuda.synchronize()
    bufs = [runtime.GBuffer.allocate(workloads.rays(v)) for v in frames]
    got = []
    for views, lt, g in zip(frames, lites, bufs):
        ctx.forward(views, g, opts)
        got.append(ctx.shade_lite(views, lt, g))
    torch.cuda.synchronize()
    for i, (a, b) in enumerate(zip(got, want)):
        np.testing.assert_array_equal(a.cpu().numpy(), b, err_msg=f"frame {i}")
