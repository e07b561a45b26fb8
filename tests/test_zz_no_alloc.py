"""nd_march_forward_noalloc: the forward march for callers that cannot allocate
device memory (a host whose allocator owns the device, a render thread where an
allocation may synchronise the device).  It runs the same persistent march as
nd_march_forward, so depth, steps, evaluation counts and hits must match exactly,
call after call.  nd_march_forward evaluates the normal taps of rays without a
shadow ray in a separate shade pass; the no-allocation path, which has no per-ray
scratch for that pass, evaluates them inside the march.  The FP32 DE compiled into
two kernels may round differently in its last bits (the compiler fuses multiplies
and adds according to each kernel's code), so normals and shade are compared within
the normal tolerance of the parity tests: p99 angle <= 2 degrees.

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test.
"""

import ctypes as C

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu

KEYS = ("depth", "steps", "shadow", "depth64", "evals")  # exact
NORMAL_DEG_P99 = 2.0
SHADE_P99 = 0.02


def _noalloc(lib):
    fn = lib.nd_march_forward_noalloc
    fn.restype = C.c_int32
    fn.argtypes = [C.POINTER(abi.nd_view_desc), C.c_int32, C.POINTER(abi.nd_march_opts),
                   C.POINTER(abi.nd_gbuffer), C.c_void_p]
    return fn


def _gbuf(n):
    g = runtime.GBuffer.allocate(n)
    g.trap = None  # the no-allocation entry point has no trap pass
    g.iters = None
    return g


def _views_single():
    fid = runtime.find_formula(workloads.MANDELBOX)
    return [abi.make_view(fid, 96, 72, (2.2, 1.3, -3.1), fov_y_deg=60.0, params=workloads.mandelbox_params(-1.5, 12),
                          max_steps=256, normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=1e-4, shadow=1,
                          light_dir=list(workloads.LIGHT_DIR))]


def _views_batched():
    return workloads.batched_64(runtime.find_formula, nviews=6, min_side=24, max_side=64, seed=11)


def test_noalloc_matches_forward_twice(ndlib):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = runtime.Context(0)
    fn = _noalloc(ndlib)
    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, refill_threshold=4)
    for views in (_views_single(), _views_batched()):
        n = workloads.rays(views)
        ref = _gbuf(n)
        ctx.forward(views, ref, opts)
        torch.cuda.synchronize()
        want = ref.numpy()
        for call in range(2):  # two calls in a row share the one scratch array
            got_buf = _gbuf(n)
            arr = (abi.nd_view_desc * len(views))(*views)
            g = got_buf.as_abi()
            st = fn(arr, len(views), C.byref(opts), C.byref(g), None)
            assert st == abi.ND_OK, abi.STATUS_NAMES[st]
            torch.cuda.synchronize()
            got = got_buf.numpy()
            for k in KEYS:
                np.testing.assert_array_equal(got[k], want[k], err_msg=f"call {call}: {k} differs")
            np.testing.assert_array_equal(got["normal"][:, 3], want["normal"][:, 3], err_msg="hit flags differ")
            hit = want["normal"][:, 3] > 0.5
            if hit.any():
                cosang = np.clip((got["normal"][hit, :3] * want["normal"][hit, :3]).sum(1), -1.0, 1.0)
                ang = np.degrees(np.arccos(cosang))
                assert np.percentile(ang, 99) <= NORMAL_DEG_P99, f"call {call}: normal p99 {np.percentile(ang, 99)}"
                dsh = np.abs(got["shade"][hit] - want["shade"][hit])
                assert np.percentile(dsh, 99) <= SHADE_P99, f"call {call}: shade p99 {np.percentile(dsh, 99)}"
    ctx.close()


def test_noalloc_rejects_what_it_cannot_serve(ndlib):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    fn = _noalloc(ndlib)
    views = _views_single()
    n = workloads.rays(views)
    full = runtime.GBuffer.allocate(n)  # trap and iters requested
    arr = (abi.nd_view_desc * 1)(*views)
    g = full.as_abi()
    assert fn(arr, 1, None, C.byref(g), None) == abi.ND_ERR_UNSUPPORTED
    too_many = (abi.nd_view_desc * 65)(*([views[0]] * 65))
    small = _gbuf(n * 65)
    g2 = small.as_abi()
    assert fn(too_many, 65, None, C.byref(g2), None) == abi.ND_ERR_INVALID


def test_noalloc_reports_a_watchdog_expiry(ndlib):
    # nd_march_forward_noalloc_stats reads the scratch array's statistics block: a
    # march stopped by a 1 ms watchdog budget comes back as ND_ERR_TIMEOUT, and the
    # next call with the default budget runs to the end again
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    fid = runtime.find_formula(workloads.MANDELBOX)
    views = [abi.make_view(fid, 512, 512, workloads.reference_initial_camera(), fov_y_deg=90.0,
                           params=workloads.mandelbox_params(-1.5, 30), max_steps=4096, eps_coef=1e-7,
                           eps_floor=0.0, normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=1e-7)]
    n = workloads.rays(views)
    fn = _noalloc(ndlib)
    stats = ndlib.nd_march_forward_noalloc_stats
    arr = (abi.nd_view_desc * 1)(*views)
    gb = _gbuf(n)
    g = gb.as_abi()
    st = abi.nd_stats()
    err = C.create_string_buffer(256)
    short = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=64, watchdog_ms=1)
    assert fn(arr, 1, C.byref(short), C.byref(g), None) == abi.ND_OK
    assert stats(None, C.byref(st), err, 256) == abi.ND_ERR_TIMEOUT
    assert st.timeouts > 0 and st.rays < n
    assert b"watchdog" in err.value
    normal = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=64)
    assert fn(arr, 1, C.byref(normal), C.byref(g), None) == abi.ND_OK
    assert stats(None, C.byref(st), err, 256) == abi.ND_OK
    assert st.timeouts == 0 and st.rays == n


def test_noalloc_refuses_stream_capture(ndlib):
    # the call copies its view table from its own stack frame, which a graph replay
    # would read after the frame is gone: on a capturing stream it enqueues nothing
    # and returns ND_ERR_UNSUPPORTED
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    fn = _noalloc(ndlib)
    views = _views_single()
    gb = _gbuf(workloads.rays(views))
    g = gb.as_abi()
    arr = (abi.nd_view_desc * 1)(*views)
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    x = torch.zeros(4, device="cuda")
    with torch.cuda.graph(graph, stream=side, capture_error_mode="relaxed"):
        status = fn(arr, 1, None, C.byref(g), C.c_void_p(side.cuda_stream))
        x += 1.0
    assert status == abi.ND_ERR_UNSUPPORTED
    graph.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
    # outside a capture the same call runs
    assert fn(arr, 1, None, C.byref(g), None) == abi.ND_OK
    torch.cuda.synchronize()
