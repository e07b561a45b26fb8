"""The persistent kernel's work list: warps take runs of consecutive ray indices from
a 64-bit counter (WarpRuns in csrc/nd_rayprog.h).  These tests run that same code on
the host with a plain counter standing in for the device atomic."""

import pytest

from numericdream_b200 import opcount

# resident warps of a full B200 launch: 148 SMs x 7 blocks x 4 warps
WARPS = 148 * 7 * 4


def check(total, warps, chunk, start, seed=1):
    s, seen = opcount.sim_work_runs(total, warps, chunk, start, seed)
    assert s["handed"] == total - start
    assert s["lowest"] == start and s["highest"] == total - 1
    assert (seen == 1).all(), "a ray index was handed out twice or never"
    assert s["counter"] >= total
    return s


def test_largest_launch_hands_out_every_ray_once():
    # the largest launch the host accepts: 2^31 - 1 rays.  Every warp adds one more
    # run after the list is used up, so the counter ends above 2^31 - 1; none of
    # those values may come back as a (negative) ray index.
    total = 2**31 - 1
    for chunk in (1, 17, 64):
        s = check(total, WARPS, chunk, start=total - 300_000, seed=chunk)
        assert s["counter"] > 2**31, "the run did not go past 2^31 (nothing exercised)"


@pytest.mark.parametrize("total,warps,chunk", [(1, 1, 1), (1, 37, 64), (1000, 37, 1), (1000, 37, 64),
                                               (65536, 4, 16), (4097, WARPS, 1)])
def test_small_launches(total, warps, chunk):
    check(total, warps, chunk, start=0, seed=total + chunk)


def test_magic_division_of_ray_indices():
    # ray_uv divides ray indices (< 2^31) by a view's pixel count and width with a
    # precomputed multiplier and shift; it must equal integer division everywhere
    import ctypes as C

    import numpy as np

    lib = opcount._load()
    lib.nd_div_by.argtypes = [C.c_uint32, C.c_int64, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(5)
    divisors = list(range(1, 3000)) + [int(x) for x in rng.integers(1, 2**31, 3000)]
    divisors += [2**k + o for k in range(31) for o in (-1, 0, 1) if 0 < 2**k + o < 2**31]
    for d in divisors:
        n = np.concatenate([rng.integers(0, 2**31, 64), [0, 1, d - 1, d, d + 1, 2**31 - 1, 2**31 - 2]])
        n = n[(n >= 0) & (n < 2**31)].astype(np.uint32)
        q = np.zeros_like(n)
        lib.nd_div_by(d, n.size, n.ctypes.data, q.ctypes.data)
        np.testing.assert_array_equal(q, n // np.uint32(d), err_msg=f"d={d}")
