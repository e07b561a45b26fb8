"""Forward calls enqueued back to back without host synchronisation (the caller
renders the next frame while the previous one runs): on one stream and alternating
between two streams, each call's G-buffer equals the same call made alone."""

import numpy as np
import pytest
import torch

from numericdream_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu

KEYS = ("depth64", "steps", "evals", "normal", "trap")


def _frames():
    return [workloads.batched_64(runtime.find_formula, nviews=8, max_side=160, seed=s) for s in (21, 22, 23, 24)]


def _alone(ctx, views):
    g = runtime.GBuffer.allocate(workloads.rays(views))
    ctx.forward(views, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    torch.cuda.synchronize()
    return g.numpy()


@pytest.mark.parametrize("two_streams", [False, True])
def test_back_to_back_forwards(ctx, two_streams):
    frames = _frames()
    want = [_alone(ctx, f) for f in frames]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()] if two_streams else [torch.cuda.Stream()]
    bufs = [runtime.GBuffer.allocate(workloads.rays(f)) for f in frames]
    torch.cuda.synchronize()
    for i, (f, g) in enumerate(zip(frames, bufs)):
        s = streams[i % len(streams)]
        ctx.forward(f, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT), stream=s.cuda_stream)
    torch.cuda.synchronize()
    for i, (g, w) in enumerate(zip(bufs, want)):
        got = g.numpy()
        for k in KEYS:
            np.testing.assert_array_equal(got[k], w[k], err_msg=f"frame {i}: {k}")
    st = ctx.stats()
    assert st.rays == workloads.rays(frames[-1]) and st.timeouts == 0


def test_rgba16f_normal_output(ctx):
    """normal_half holds the f32 normal rounded to IEEE halves (w = hit), as the
    reference's RGBA16F normal target."""
    views = _frames()[0]
    n = workloads.rays(views)
    g = runtime.GBuffer.allocate(n)
    g.normal_half = torch.empty((n, 4), dtype=torch.float16, device="cuda")
    ctx.forward(views, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT))
    out = g.numpy()
    np.testing.assert_array_equal(out["normal_half"].view(np.uint16), out["normal"].astype(np.float16).view(np.uint16))


def test_measured_fp32_peak(ctx):
    """nd_measure_fp32_peak lands near the nominal FP32 FMA rate (148 SMs x 128 lanes x
    2 FLOP x clock: 74.4 TFLOP/s at 1965 MHz)."""
    tf = ctx.measure_fp32_peak(10.0)
    print("measured FP32 peak", tf, "TFLOP/s")
    assert 40.0 < tf < 80.0
