"""The autotuner's cache file (nd_tune_cache_save / nd_tune_cache_load) without a GPU:
entries read from JSON come back out of a save with the same keys and values, keys of
any length and with characters JSON must escape survive the round trip, and entries
the library cannot use (an unknown kernel, block size or refill threshold) are skipped."""

import json

import pytest

from numericdream_b200 import runtime


def test_cache_round_trip_and_invalid_entries(ndlib, tmp_path):
    long_key = "B200 | " + "|".join(f"formula_{i:03d}" for i in range(60)) + " | 0123456789abcdef"
    good = [
        {"key": "NVIDIA B200 | mandelbrot | 00ff", "kernel": 2, "block": 64, "blocks_per_sm": 14,
         "refill_threshold": 6, "rays_per_s": 1.0e9},
        {"key": long_key, "kernel": 1, "block": 128, "blocks_per_sm": 0, "refill_threshold": 1, "rays_per_s": 2.0e8},
        {"key": 'quote " backslash \\ tab \t end', "kernel": 2, "block": 256, "blocks_per_sm": -2,
         "refill_threshold": 12, "rays_per_s": 5.5e8},
    ]
    bad = [
        {"key": "bad kernel", "kernel": 9, "block": 128, "blocks_per_sm": 0, "refill_threshold": 6},
        {"key": "bad block", "kernel": 2, "block": 96, "blocks_per_sm": 0, "refill_threshold": 6},
        {"key": "bad threshold", "kernel": 2, "block": 128, "blocks_per_sm": 0, "refill_threshold": 40},
        {"kernel": 2, "block": 128},
    ]
    src = tmp_path / "in.json"
    src.write_text(json.dumps(good + bad))
    assert runtime.Context.tune_cache_load(str(src)) == len(good)
    out = tmp_path / "out.json"
    runtime.Context.tune_cache_save(str(out))
    saved = {e["key"]: e for e in json.loads(out.read_text())}
    for e in good:
        assert e["key"] in saved, e["key"][:40]
        s = saved[e["key"]]
        for k in ("kernel", "block", "blocks_per_sm", "refill_threshold"):
            assert s[k] == e[k], (e["key"][:40], k)
        assert s["rays_per_s"] == pytest.approx(e["rays_per_s"], rel=1e-5)
    for e in bad:
        assert e.get("key") not in saved
    # a file that is not a JSON array of entries is refused; a missing file is not found
    (tmp_path / "broken.json").write_text("{not json")
    with pytest.raises(runtime.NDError):
        runtime.Context.tune_cache_load(str(tmp_path / "broken.json"))
    with pytest.raises(runtime.NDError):
        runtime.Context.tune_cache_load(str(tmp_path / "missing.json"))
