"""Comparison of G-buffers from the CUDA library against the CPU oracle."""

from __future__ import annotations

import numpy as np


def compare(gpu: dict, ref: dict, mask=None) -> dict:
    """Statistics of one G-buffer against an oracle run of the same rays; the
    depth/normal/trap errors are taken over rays both hit (and inside mask)."""
    gh = gpu["normal"][:, 3] > 0.5
    rh = ref["normal"][:, 3] > 0.5
    both = gh & rh
    if mask is not None:
        both = both & mask
    out = {"rays": int(gh.size), "hits_gpu": int(gh.sum()), "hits_ref": int(rh.sum()),
           "hit_mismatch": int((gh != rh).sum()),
           "steps_mismatch": int((gpu["steps"].astype(np.int64) != ref["steps"].astype(np.int64)).sum()),
           "iters_mismatch": int(((gpu["iters"].astype(np.int64) != ref["iters"].astype(np.int64)) & both).sum())}
    if both.any():
        d_ref = ref["depth64"][both]
        d_gpu = gpu["depth64"][both]
        rel = np.abs(d_gpu - d_ref) / np.maximum(np.abs(d_ref), 1e-30)
        out["depth_rel_max"] = float(rel.max())
        out["depth_rel_p99"] = float(np.percentile(rel, 99))
        out["depth_rel_over_1e-4"] = float((rel > 1e-4).mean())
        n_g = gpu["normal"][both, :3].astype(np.float64)
        n_r = ref["normal"][both, :3].astype(np.float64)
        cosang = np.clip((n_g * n_r).sum(1) / np.maximum(np.linalg.norm(n_g, axis=1) * np.linalg.norm(n_r, axis=1), 1e-30), -1, 1)
        ang = np.degrees(np.arccos(cosang))
        out["normal_deg_max"] = float(ang.max())
        out["normal_deg_p99"] = float(np.percentile(ang, 99))
        tr = np.abs(gpu["trap"][both].astype(np.float64) - ref["trap"][both].astype(np.float64))
        out["trap_abs_p99"] = float(np.percentile(tr, 99))
        out["trap_abs_max"] = float(tr.max())
    return out


# Boundary-case policy for the integer outputs (hit/miss, probe steps, iterations).
# A ray is "stable" when its FP64 oracle outcome is unchanged with every DE value
# scaled by 1 - 1e-4 and by 1 + 1e-4 (above the relative error of an FP32 DE), and
# "short" when its FP64 march ends within SHORT_STEPS probe steps.  Stable short
# rays must agree ray for ray.  Longer marches through chaotic fractals (rays that
# wander through an infinite lattice for hundreds of steps) amplify rounding until
# the outcome is decided by it; for those only aggregate statistics are compared.
SHORT_STEPS = 64


def policy_check(gpu: dict, base64: dict, unstable, max_strict_frac=0.001, agg_tol=0.02):
    gh = gpu["normal"][:, 3] > 0.5
    bh = base64["normal"][:, 3] > 0.5
    mism = (gh != bh) | (gpu["steps"].astype(np.int64) != base64["steps"].astype(np.int64))
    strict = (~unstable) & (base64["steps"] <= SHORT_STEPS)
    n = gh.size
    out = {"rays": n, "strict_rays": int(strict.sum()), "strict_mismatch": int((mism & strict).sum()),
           "unstable_frac": float(unstable.mean()), "all_mismatch": int(mism.sum()),
           "hit_frac_gpu": float(gh.mean()), "hit_frac_f64": float(bh.mean()),
           "mean_steps_gpu": float(gpu["steps"].mean()), "mean_steps_f64": float(base64["steps"].mean())}
    ok = out["strict_mismatch"] <= max_strict_frac * max(out["strict_rays"], 1) + 1
    ok &= abs(out["hit_frac_gpu"] - out["hit_frac_f64"]) <= agg_tol
    ok &= abs(out["mean_steps_gpu"] - out["mean_steps_f64"]) <= agg_tol * max(out["mean_steps_f64"], 1.0)
    out["ok"] = bool(ok)
    out["strict_mask"] = strict
    return out
