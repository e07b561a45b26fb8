"""Algorithmic FP32 operation counts of a launch (for the roofline numerator).

The host library libnd_opcount.so runs the same ray program and the same
translated formula code as the CUDA kernels with a counting float type, over an
even sample of each view's rays, and reports FLOPs (add + mul + div + 2 fma),
SFU calls (transcendentals and square roots) and other FP ops (compares,
min/max, abs, floor/round, selects) per DE evaluation.
"""

from __future__ import annotations

import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

SM_COUNT_B200 = 148
FP32_LANES_PER_SM = 128


def _load():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libnd_opcount.so")
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: build it with `python -m numericdream_b200.build`")
        _lib = C.CDLL(path)
        _lib.nd_opcount.argtypes = [C.POINTER(abi.nd_view_desc), C.c_int, C.c_int64, C.POINTER(C.c_double)]
        _lib.nd_opcount.restype = C.c_int
    return _lib


def count(views, rays_per_view: int = 256) -> dict:
    arr = (abi.nd_view_desc * len(views))(*views)
    out = (C.c_double * 9)()
    rc = _load().nd_opcount(arr, len(views), rays_per_view, out)
    if rc != 0:
        raise ValueError("unknown formula id in the views")
    keys = ["flops", "sfu", "other", "de_evals", "add", "mul", "div", "fma", "rays"]
    return {k: out[i] for i, k in enumerate(keys)}


def flops_per_eval_for(views, rays_per_view: int = 256):
    c = count(views, rays_per_view)
    ev = max(c["de_evals"], 1.0)
    per = {k: c[k] / ev for k in ("flops", "sfu", "other", "add", "mul", "div", "fma")}
    per["evals_per_ray"] = c["de_evals"] / max(c["rays"], 1.0)
    return per["flops"], per


def fp32_peak_tflops(sm_mhz=None, sms: int = SM_COUNT_B200) -> float:
    """Nominal FP32 FMA peak: SMs x 128 lanes x 2 FLOPs x SM clock."""
    mhz = float(sm_mhz) if sm_mhz else 1965.0
    return sms * FP32_LANES_PER_SM * 2 * mhz * 1e6 / 1e12


def sim_work_runs(total: int, warps: int, chunk: int, start: int = 0, seed: int = 1):
    """The persistent kernel's work-list bookkeeping (WarpRuns) run on the host with a
    plain counter in place of the device atomic.  Returns (summary dict, per-ray count
    of how often each index in [start, total) was handed out)."""
    import numpy as np

    lib = _load()
    if not hasattr(lib, "_sim_ready"):
        lib.nd_sim_work_runs.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_uint64, C.c_void_p,
                                         C.POINTER(C.c_int64)]
        lib.nd_sim_work_runs.restype = C.c_int
        lib._sim_ready = True
    seen = np.zeros(max(total - start, 0), dtype=np.uint8)
    out = (C.c_int64 * 5)()
    lib.nd_sim_work_runs(total, warps, chunk, start, seed, seen.ctypes.data if seen.size else None, out)
    keys = ["handed", "lowest", "highest", "counter", "claims"]
    return {k: int(out[i]) for i, k in enumerate(keys)}, seen
