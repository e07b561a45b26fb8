"""The persistent kernel's device watchdog (nd_march_opts.watchdog_ms).  A march that
runs past its deadline stops by itself (every warp reads the global timer every 64
passes and leaves its loop), the call reports ND_ERR_TIMEOUT through nd_last_stats
with the number of stopped warps, and the context stays usable: a forward with the
default budget afterwards gives the same bits as one before.  Nothing faults or
hangs: the kernel returns on its own."""

import ctypes as C

import numpy as np
import pytest

from numericdream_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu


def heavy_views(size=512):
    # Mandelbox, 30 iterations, FP64 DE, eps 1e-7 t and up to 4096 steps: tens of
    # milliseconds per call, far beyond a 1 ms budget
    fid = runtime.find_formula(workloads.MANDELBOX)
    return [abi.make_view(fid, size, size, workloads.reference_initial_camera(), fov_y_deg=90.0,
                          params=workloads.mandelbox_params(-1.5, 30), max_steps=4096, eps_coef=1e-7,
                          eps_floor=0.0, normal_mode=abi.ND_NORMAL_CENTRAL, normal_h_coef=1e-7)]


def test_watchdog_expiry_is_reported_and_the_context_recovers(ctx):
    import torch

    views = heavy_views()
    n = workloads.rays(views)
    normal = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=64)
    short = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=64, watchdog_ms=1)

    before = runtime.GBuffer.allocate(n)
    ctx.forward(views, before, normal)
    s0 = ctx.stats()
    assert s0.timeouts == 0 and s0.rays == n

    cut = runtime.GBuffer.allocate(n)
    ctx.forward(views, cut, short)
    st = abi.nd_stats()
    status = ctx.lib.nd_last_stats(ctx.handle, C.byref(st))
    assert status == abi.ND_ERR_TIMEOUT, abi.STATUS_NAMES[status]
    assert st.timeouts > 0
    assert st.rays < n, "the watchdog stopped nothing"
    assert "watchdog" in ctx.last_error()
    with pytest.raises(runtime.NDError) as e:
        ctx.stats()
    assert e.value.status == abi.ND_ERR_TIMEOUT

    after = runtime.GBuffer.allocate(n)
    ctx.forward(views, after, normal)
    s2 = ctx.stats()
    assert s2.timeouts == 0 and s2.rays == n
    torch.cuda.synchronize()
    a, b = before.numpy(), after.numpy()
    for k in ("depth", "depth64", "steps", "evals", "normal", "trap", "iters", "shade"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
