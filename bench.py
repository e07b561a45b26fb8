"""Benchmark of the B200 sphere-tracing pass.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched_64|mandelbox_1080p|mandelbulb_256]

A step is one forward march over the whole workload.  The default workload is the
batched one: 64 views of mixed formulas (Mandelbulb, Mandelbox, Menger,
pseudo-Kleinian) and uneven sizes (log-uniform 64..1024 per side, 7.2 M rays) in one
persistent launch plus the surface pass (normals, orbit trap), autotuned and replayed
as a CUDA graph.  The plain per-view launch of the same views is timed beside it, and
the 1080p x 4 spp Mandelbox frame with shadow rays is timed as a second workload.
Rank 0 prints one JSON line.

value         rays/s of the batched persistent march, device time (CUDA events on the
              launching stream), inputs resident; L2 is flushed between steps.
e2e           the same metric through the public C ABI call (nd_march_forward) with
              host view descriptors, and the G-buffer read back to pinned host memory
              every step (two G-buffers: a frame's read-back overlaps the next march;
              at least 20 frames, the last read-back inside the timed region).
roofline      FP32-pipe roofline of the march kernel: algorithmic FLOPs per launch
              (DE evaluations x FLOPs per evaluation, counted by running the same ray
              program and formula code on the host with a counting float) / kernel
              time, against the FP32 FMA peak measured on the GPU in the same run
              (nominal at the sampled SM clock if that fails); DRAM traffic and the
              issue-slot share from the committed ncu captures.
cpu_baseline  the reference's own march code compiled for the host (see below), FP32,
              on every host core over a bounded, seeded sample of the workload's rays,
              with the oracle's FP32 restatement beside it; the oracle's FP64 run on
              sampled rays gives the error figures against the GPU's output.

--impl reference times the CPU implementation of the path on the host cores: the
reference app itself only runs through WebGPU, which this machine cannot run, so its
own march code (march_to and estimate_normal of its shader template, translated
mechanically and compiled for the host into oracle/_ref) is timed in FP32 with every
host thread; where that library was not built, the oracle's FP32 restatement.
"""

from __future__ import annotations

import argparse
import json
import os
import random
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mrays/s & DE-evals/s on 1 B200, batched vs plain, at stated FP64 error"

# DRAM bytes (read + write) of one forward's kernels on each workload, from
# ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum (one capture per workload;
# the summary and its command are in profiles/).
NCU_TRAFFIC = {"batched_64": {"march": 307.5e6, "surface": 391.7e6},
               "mandelbox_1080p": {"march": 321.1e6, "surface": 499.8e6, "shadow": 330.3e6}}
# The march kernel's share of issue slots busy on batched_64 (ncu --set full, one
# capture; the summary and its command are in profiles/).
NCU_ISSUE = {"batched_64": 0.865}


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while the timed work runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
            except (ValueError, IndexError):
                continue
            for i, n in enumerate(self.NAMES):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_views(name, resolve, world=1, rank=0, names=None):
    """The workload's views; with world > 1, rank `rank`'s share of the one batch
    (views cut into tiles and balanced over the ranks: numericdream_b200.shard)."""
    from numericdream_b200 import shard, workloads

    if name == "batched_64":
        views = workloads.batched_64(resolve, seed=7)
    elif name == "mandelbox_1080p":
        views = workloads.mandelbox_1080p(resolve, seed=1234)
    elif name == "mandelbulb_256":
        views = workloads.mandelbulb_256(resolve)
    else:
        raise SystemExit(f"unknown workload {name}")
    return shard.rank_views(views, world, rank, names) if world > 1 else views


def config_of(name, views, ws, rays_total=None):
    from numericdream_b200 import workloads

    c = {"workload": name, "views": len(views), "rays_per_step": rays_total or workloads.rays(views),
         "max_steps": int(max(v.max_steps for v in views)), "de": "fp32 (fast math)", "t": "fp64",
         "l2": "flushed between steps (256 MiB write)", "parallelism": f"shards{ws}" if ws > 1 else "single"}
    if ws > 1:
        c["sharding"] = ("one batch per step, its views cut into tiles and balanced over the ranks "
                         "(longest-processing-time first); rank 0's share: %d tiles" % len(views))
    return c


def cpu_sample(views, target_rays, seed=0, run=64):
    """Seeded runs of `run` consecutive rays spread over every view: (view index, first, n)."""
    from numericdream_b200 import abi

    rng = random.Random(seed)
    total = sum(abi.rays_of(v) for v in views)
    frac = min(1.0, target_rays / max(total, 1))
    out = []
    for i, v in enumerate(views):
        n = abi.rays_of(v)
        runs = max(1, int(n * frac) // run)
        for _ in range(runs):
            first = rng.randrange(0, max(1, n - run))
            out.append((i, first, min(run, n - first)))
    return out


def run_cpu(views, seconds_budget=15.0, with_fp64=False, names=None):
    """The oracle's FP32 march on all host cores over a bounded sample (timed), and
    optionally the FP64 oracle on the same sample (for the error figures).  names:
    formula names by id (default: the CUDA library's registry)."""
    from oracle import pyoracle

    cores = pyoracle.max_threads()
    if names is None:
        from numericdream_b200 import runtime

        names = runtime.formula_names()
    names = [names[v.formula] for v in views]
    t0 = time.perf_counter()
    nr = 0
    for vi, first, n in cpu_sample(views, 2048, seed=1):
        pyoracle.render(views[vi], names[vi], precision=32, first=first, n=n)
        nr += n
    rate = nr / max(time.perf_counter() - t0, 1e-6)
    chunks = cpu_sample(views, max(int(rate * seconds_budget), 4096), seed=2)
    t0 = time.perf_counter()
    rays = evals = 0
    for vi, first, n in chunks:
        o = pyoracle.render(views[vi], names[vi], precision=32, first=first, n=n)
        rays += n
        evals += int(o["evals"].astype("int64").sum())
    dt = time.perf_counter() - t0
    res = {"rays_per_s": rays / dt, "evals_per_s": evals / dt, "rays": rays, "seconds": dt, "cores": cores,
           "chunks": chunks}
    if with_fp64:
        res["fp64"] = [pyoracle.render(views[vi], names[vi], precision=64, first=first, n=n)
                       for vi, first, n in chunks[: max(1, len(chunks) // 4)]]
    return res


def reference_lib():
    """oracle/_ref's library (the reference's own march, compiled for the host), or None
    where it was not built (it needs the reference's sources at build time)."""
    import ctypes as C

    path = os.path.join(ROOT, "oracle", "_ref", "libref_formulas.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    if not hasattr(lib, "ref_trace"):
        return None
    lib.ref_trace.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int64, C.c_int64, C.c_void_p]
    lib.ref_trace.restype = C.c_int
    return lib


def run_cpu_reference(lib, views, seconds_budget=15.0, names=None):
    """The reference's own fs_simple primary pass (march_to and estimate_normal of its
    shader template, translated mechanically and compiled for the host; FP32 like the
    reference) on all host cores over a bounded, seeded sample of the views' rays.
    names: formula names by id (default: the CUDA library's registry)."""
    import ctypes as C

    import numpy as np

    from oracle import pyoracle

    cores = pyoracle.max_threads()
    if names is None:
        from numericdream_b200 import runtime

        names = runtime.formula_names()
    names = [names[v.formula].encode() for v in views]

    def run(chunks):
        rays = evals = 0
        for vi, first, n in chunks:
            out = np.zeros((n, 12))
            if lib.ref_trace(C.addressof(views[vi]), names[vi], 32, first, n, out.ctypes.data) != 0:
                raise RuntimeError(f"no reference march for {names[vi]!r}")
            rays += n
            evals += int(out[:, 3].sum() + out[:, 7].sum())
        return rays, evals

    t0 = time.perf_counter()
    r0, _ = run(cpu_sample(views, 2048, seed=1))
    rate = r0 / max(time.perf_counter() - t0, 1e-6)
    chunks = cpu_sample(views, max(int(rate * seconds_budget), 4096), seed=2)
    t0 = time.perf_counter()
    rays, evals = run(chunks)
    dt = time.perf_counter() - t0
    return {"rays_per_s": rays / dt, "evals_per_s": evals / dt, "rays": rays, "seconds": dt, "cores": cores}


def sampled_errors(views, gbuf, target_rays, seed, names=None, run=64, de_precision=64, min_t=1e-3, chunks=None):
    """The G-buffer (device tensors) against the FP64 oracle on seeded runs of `run`
    consecutive rays over every view (about target_rays rays): the same statistics
    as error_stats, plus the oracle's time.  Only the sampled slices are copied."""
    import numpy as np

    from numericdream_b200 import abi
    from oracle import pyoracle

    if names is None:
        from numericdream_b200 import runtime

        names = runtime.formula_names()
    offs = [0]
    for v in views:
        offs.append(offs[-1] + abi.rays_of(v))
    if chunks is None:
        chunks = cpu_sample(views, target_rays, seed=seed, run=run)
    t0 = time.perf_counter()
    refs, gpus = [], []
    for vi, first, cnt in chunks:
        refs.append(pyoracle.render(views[vi], names[views[vi].formula], precision=de_precision, first=first, n=cnt))
        sl = slice(offs[vi] + first, offs[vi] + first + cnt)
        gpus.append({"normal": gbuf.normal[sl].cpu().numpy(), "depth64": gbuf.depth64[sl].cpu().numpy()})
    dt = time.perf_counter() - t0
    out = error_stats(views, None, {"chunks": chunks, "fp64": refs}, gpu_parts=gpus, min_t=min_t)
    out["oracle_seconds"] = dt
    return out


def deepzoom_normal_floor(views, target_rays, seed):
    """The FP64 oracle's own normal noise at the deep-zoom camera: the angle between its
    normals and those of the same oracle compiled with fused multiply-adds (results
    that differ by rounding only), on the same sampled rays."""
    import numpy as np

    from numericdream_b200 import runtime
    from oracle import pyoracle

    names = runtime.formula_names()
    angles = []
    for vi, first, cnt in cpu_sample(views, target_rays, seed=seed):
        v = views[vi]
        a = pyoracle.render(v, names[v.formula], precision=64, first=first, n=cnt)
        b = pyoracle.render(v, names[v.formula], precision=64, first=first, n=cnt, fma=True)
        both = (a["normal"][:, 3] > 0.5) & (b["normal"][:, 3] > 0.5)
        x, y = a["normal"][both, :3].astype(np.float64), b["normal"][both, :3].astype(np.float64)
        c = (x * y).sum(1) / np.maximum(np.linalg.norm(x, axis=1) * np.linalg.norm(y, axis=1), 1e-300)
        angles.append(np.degrees(np.arccos(np.clip(c, -1.0, 1.0))))
    ang = np.concatenate(angles) if angles else np.zeros(1)
    return {"normal_deg_p50": float(np.percentile(ang, 50)), "normal_deg_p99": float(np.percentile(ang, 99)),
            "note": "FP64 oracle against the same oracle compiled with FMA contraction, same sampled rays"}


def error_stats(views, gbuf_np, cpu, gpu_parts=None, min_t=1e-3):
    """GPU output against the FP64 oracle on the sampled rays (hits of both, beyond
    t = min_t)."""
    import numpy as np

    from numericdream_b200 import abi

    offs = [0]
    for v in views:
        offs.append(offs[-1] + abi.rays_of(v))
    rel, ang, mism, n = [], [], 0, 0
    for k, ((vi, first, cnt), ref) in enumerate(zip(cpu["chunks"], cpu["fp64"])):
        if gpu_parts is not None:
            gn, gd = gpu_parts[k]["normal"], gpu_parts[k]["depth64"]
        else:
            sl = slice(offs[vi] + first, offs[vi] + first + cnt)
            gn, gd = gbuf_np["normal"][sl], gbuf_np["depth64"][sl]
        gh = gn[:, 3] > 0.5
        rh = ref["normal"][:, 3] > 0.5
        mism += int((gh != rh).sum())
        n += cnt
        both = gh & rh & (ref["depth64"] > min_t)
        if both.any():
            rel.append(np.abs(gd[both] - ref["depth64"][both]) / ref["depth64"][both])
            a = gn[both, :3].astype(np.float64)
            b = ref["normal"][both, :3].astype(np.float64)
            c = np.clip((a * b).sum(1) / np.maximum(np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1), 1e-30), -1, 1)
            ang.append(np.degrees(np.arccos(c)))
    rel = np.concatenate(rel) if rel else np.zeros(1)
    ang = np.concatenate(ang) if ang else np.zeros(1)
    return {"sample_rays": n, "hit_mismatch_frac": mism / max(n, 1),
            "depth_rel_p99": float(np.percentile(rel, 99)), "depth_rel_max": float(rel.max()),
            "depth_rel_frac_over_1e-4": float((rel > 1e-4).mean()),
            "normal_deg_p99": float(np.percentile(ang, 99)), "normal_deg_max": float(ang.max()),
            "note": f"all sampled rays incl. rounding-unstable ones; hits with t > {min_t:g}"}


def build_manifest_names():
    """Formula names in formula-id order, from the build's manifest (the CUDA library
    numbers its formulas in this order), so that the reference arm resolves names
    without loading the CUDA library."""
    path = os.path.join(ROOT, "numericdream_b200", "_generated", "manifest.json")
    with open(path) as fh:
        return json.load(fh)["formulas"]


def reference_arm(args):
    ws, rank, _ = _dist_env()
    if rank != 0:
        return 0
    try:
        names = build_manifest_names()
    except (OSError, ValueError, KeyError) as e:
        print(json.dumps({"impl": "reference", "unavailable": f"formula table not built: {e}"}))
        return 0
    views = build_views(args.workload, names.index)
    per, res = [], None
    budget = max(2.0, 60.0 / max(args.steps + args.warmup, 1))
    ref = reference_lib()
    t_all = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        if ref:
            res = run_cpu_reference(ref, views, seconds_budget=budget, names=names)
        else:
            res = run_cpu(views, seconds_budget=budget, names=names)
        if i >= args.warmup:
            per.append(res)
            t_all.append(time.perf_counter() - t0)
    v = sum(r["rays_per_s"] for r in per) / len(per) / 1e6
    if ref:
        kind = "reference"
        note = ("the reference's own fs_simple pass (march_to and estimate_normal of its shader template, "
                "translated mechanically and compiled for the host by oracle/build_ref.py), FP32 as in the "
                "reference, all host threads; the reference app itself runs only through WebGPU, unavailable "
                "on this box")
    else:
        kind = "port"
        note = ("the reference's march restated on the CPU (FP32, all host threads); the reference app itself "
                "runs only through WebGPU, unavailable on this box")
    # a step is one bounded sample of the workload: its wall time, and the whole
    # workload's time at the measured rate
    line = {"metric": METRIC, "value": v, "unit": "Mrays/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(r["rays"] for r in per) / len(per) / (v * 1e6),
            "sample_wall_ms_per_step": 1e3 * sum(t_all) / len(t_all), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded views, no dataset)",
            "config": config_of(args.workload, views, 1),
            "de_evals_per_s": sum(r["evals_per_s"] for r in per) / len(per),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": res["cores"], "kind": kind,
                             "sample": f"{res['rays']} rays per step in seeded runs of 64 over all views"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": note}
    print(json.dumps(line))
    return 0


def profile_forward(args):
    """One forward of the workload (persistent march + shade pass) for a profiler;
    with --repeat N, N more forwards after it, reporting the median of the march
    kernel's CUDA-event times (L2 flushed before each)."""
    import torch

    from numericdream_b200 import abi, runtime, workloads

    ctx = runtime.Context(0)
    views = build_views(args.workload, runtime.find_formula)
    if args.views_of:
        views = [v for v in views if runtime.formula_name(v.formula) == args.views_of]
        if not views:
            raise SystemExit(f"no view of {args.views_of} in {args.workload}")
    for v in views:
        if args.accel_res:
            v.accel_res, v.accel_levels, v.accel_safety = args.accel_res, 6, 0.92
        if args.formula:
            # the same cameras against another formula at its @param defaults (with
            # sphere_primitive: the cost of the ray program around a one-step DE)
            v.formula = runtime.find_formula(args.formula)
            defaults = [p.default_value for p in runtime.formula_params(v.formula)]
            for i in range(16):
                v.params[i] = defaults[i] if i < len(defaults) else 0.0
    g = runtime.GBuffer.allocate(workloads.rays(views))
    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, refill_threshold=4)
    ctx.forward(views, g, opts)
    march_ms = []
    if args.repeat > 0:
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        for _ in range(args.repeat):
            flush.fill_(1)
            ctx.forward(views, g, opts)
            march_ms.append(ctx.stats().march_ms)
    if args.with_lite:
        lite = abi.make_lite([((0.05, 0.05, 0.22), 0.0, 0.2, 1.3), ((1.0, 0.95, 0.82), 1.0, 0.8, 1.7)],
                             [(abi.ND_LIGHT_GLOBAL, (0.4, 0.8, -0.45), (1.0, 0.95, 0.9), 1.2)])
        ctx.shade_lite(views, [lite] * len(views), g)
    torch.cuda.synchronize()
    st = ctx.stats()
    line = {"workload": args.workload, "views": len(views), "rays": workloads.rays(views), "de_evals": st.de_evals,
            "march_evals": st.march_evals, "normal_evals": st.normal_evals, "hits": st.hits}
    if march_ms:
        m = sorted(march_ms)[len(march_ms) // 2]
        line.update({"march_ms_median": m, "sm_ns_per_march_eval": m * 1e6 * torch.cuda.get_device_properties(0).multi_processor_count
                                              / max(st.march_evals, 1)})
    print(json.dumps(line))
    ctx.close()
    return 0


def small_and_deepzoom(ctx, sptr, timed, steps, with_errors=True):
    """The single-view Mandelbulb 256x256 (persistent and plain) and the deep-zoom frame
    (Mandelbox, 30 iterations, 4096x4096 in 16 tiles of 1024x1024, FP64 DE), each with
    its depth and normal error against the FP64 oracle."""
    import torch

    from numericdream_b200 import abi, runtime, workloads

    out = {}
    v = workloads.mandelbulb_256(runtime.find_formula)
    n = workloads.rays(v)
    g = runtime.GBuffer.allocate(n)
    # "auto": the default options, which run the plain launch for one view that fits in
    # one round of the persistent grid
    for label, kern in (("persistent", abi.ND_KERNEL_PERSISTENT), ("plain", abi.ND_KERNEL_PLAIN),
                        ("auto", abi.ND_KERNEL_AUTO)):
        o = runtime.make_opts(kernel=kern)
        ms = timed(lambda: ctx.forward(v, g, o, stream=sptr), steps, 3)
        out[f"mandelbulb_256_{label}"] = {"ms_per_step": ms, "Mrays_per_s": n / (ms * 1e-3) / 1e6}
        if label == "auto":
            out["mandelbulb_256_auto"]["kernel"] = "plain" if ctx.stats().kernel == abi.ND_KERNEL_PLAIN else "persistent"
        if label == "persistent" and with_errors:
            torch.cuda.synchronize()
            # every ray of the view against the FP64 oracle
            out["mandelbulb_256_persistent"]["error_vs_fp64"] = sampled_errors(v, g, 0, 0, chunks=[(0, 0, n)])
    views = workloads.deepzoom_4096(runtime.find_formula, ctx)
    n = workloads.rays(views)
    g = runtime.GBuffer.allocate(n)
    o = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=64)
    ms = timed(lambda: ctx.forward(views, g, o, stream=sptr), 1, 1)
    st = ctx.stats()
    out["deepzoom_4096"] = {"ms_per_frame": ms, "Mrays_per_s": n / (ms * 1e-3) / 1e6,
                            "de_evals_per_s": st.de_evals / (ms * 1e-3), "hits": st.hits, "rays": n,
                            "de": "fp64 (an FP32 DE cannot resolve the 1e-12 pixel footprint: no ray hits)"}
    if with_errors:
        torch.cuda.synchronize()
        # hits lie at t ~ 1e-5 here: no t floor
        out["deepzoom_4096"]["error_vs_fp64"] = sampled_errors(views, g, 8192, 5, min_t=0.0)
        out["deepzoom_4096"]["normal_noise_floor"] = deepzoom_normal_floor(views, 8192, 5)
    # lite shading (shade_lite) of batched_64's hits after each forward: colour strip,
    # ambient occlusion (5 DE evaluations per hit), two lights
    views = workloads.batched_64(runtime.find_formula)
    n = workloads.rays(views)
    g = runtime.GBuffer.allocate(n)
    o = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT)
    stops = [((0.05, 0.05, 0.22), 0.0, 0.2, 1.3), ((0.85, 0.35, 0.08), 0.5, 0.5, 1.5), ((1.0, 0.95, 0.82), 1.0, 0.8, 1.7)]
    lights = [(abi.ND_LIGHT_GLOBAL, (0.4, 0.8, -0.45), (1.0, 0.95, 0.9), 1.2),
              (abi.ND_LIGHT_POINT, (2.0, 2.5, -3.0), (0.6, 0.7, 1.0), 6.0)]
    lites = [abi.make_lite(stops, lights) for _ in views]
    ms_fwd = timed(lambda: ctx.forward(views, g, o, stream=sptr), steps, 3)
    ms_lite = timed(lambda: (ctx.forward(views, g, o, stream=sptr), ctx.shade_lite(views, lites, g, stream=sptr)),
                    steps, 3)
    out["batched_64_lite"] = {"ms_per_step": ms_lite, "Mrays_per_s": n / (ms_lite * 1e-3) / 1e6,
                              "lite_pass_ms": ms_lite - ms_fwd,
                              "note": "forward + nd_shade_lite (colour strip, AO, 2 lights) per step"}
    # batched_64 with the empty-space accelerator on: the reference's default grid
    # (64^3 x 6 cascades, safety 0.92) and a coarse one; grids built inside every step
    for res in (64, 16):
        av = []
        for v in views:
            w = abi.nd_view_desc.from_buffer_copy(v)
            w.accel_res, w.accel_levels, w.accel_safety = res, 6, 0.92
            av.append(w)
        ms = timed(lambda: ctx.forward(av, g, o, stream=sptr), steps, 3)
        st = ctx.stats()
        out[f"batched_64_accel_{res}"] = {"ms_per_step": ms, "Mrays_per_s": n / (ms * 1e-3) / 1e6,
                                          "march_evals": st.march_evals, "grid_cells": st.accel_voxels,
                                          "grid_build_ms": st.accel_ms, "march_ms": st.march_ms,
                                          "hits": st.hits}
    return out


def differentiation_step(ctx, stream, sptr, timed, steps):
    """Differentiation workload: 16 problems of a 512x512 Mandelbulb (Lambert, one
    light, orbit camera); one step = the FP32 forward of the 16 start views, dLoss/dshade
    of the mean-L2 loss to the targets, and the adjoint for (power, bailout, yaw, pitch,
    dist).  The targets are rendered once, outside the timed region."""
    import torch

    from numericdream_b200 import abi, runtime, workloads

    sv, sc, tv, _ = workloads.differentiation_16(runtime.find_formula)
    n = workloads.rays(sv)
    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT)
    gt = runtime.GBuffer.allocate(n)
    ctx.forward(tv, gt, opts, stream=sptr)
    g = runtime.GBuffer.allocate(n)
    stream.synchronize()
    target = gt.shade.clone()
    out = {"workload": "differentiation_16 (16 x 512x512 Mandelbulb, Lambert, orbit camera)",
           "rays_per_step": n}
    for prec in (32, 64):
        def step():
            ctx.forward(sv, g, opts, stream=sptr)
            dl = (2.0 / n) * (g.shade - target)
            ctx.backward(sv, sc, g, dl, param_idx=(0, 2), de_precision=prec, stream=sptr)

        ms = timed(step, steps, 2)
        out[f"ms_per_step_adjoint_fp{prec}"] = ms
        out[f"rays_per_s_adjoint_fp{prec}"] = n / (ms * 1e-3)
    ms_f = timed(lambda: ctx.forward(sv, g, opts, stream=sptr), steps, 2)
    out["ms_forward"] = ms_f
    out["note"] = ("forward + adjoint per step; the adjoint spends 3 + 6 + 7 x 5 dual-number DE evaluations "
                   "per hit ray (gradient, normal taps, then per theta the hit and six taps)")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched_64")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the second (1080p Mandelbox) workload")
    ap.add_argument("--with-lite", action="store_true", help="--profile-forward: also one lite shading pass")
    ap.add_argument("--accel-res", type=int, default=0, help="--profile-forward: accelerator grids of this size")
    ap.add_argument("--formula", default="", help="--profile-forward: every view's formula replaced by this one")
    ap.add_argument("--views-of", default="", help="--profile-forward: only the views of this formula")
    ap.add_argument("--repeat", type=int, default=0, help="--profile-forward: timed forwards after the first")
    ap.add_argument("--profile-forward", action="store_true",
                    help="run ONE forward of the workload through the public API and exit (for ncu captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ and not args.profile_forward:
        # one process per GPU: start the ranks under torch.distributed.run
        import socket

        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
        return subprocess.call(cmd)
    if args.profile_forward:
        return profile_forward(args)

    import numpy as np
    import torch

    from numericdream_b200 import abi, runtime, workloads

    ws, rank, local = _dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        if ws != args.gpus and rank == 0:
            print(f"note: --gpus {args.gpus} but WORLD_SIZE {ws}; running {ws} ranks", file=sys.stderr)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = runtime.Context(local)
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(fn, steps, warmup):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                fn()
        stream.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        return total / steps

    def over_ranks(times, counts):
        """Times: the max over ranks; counts: the sum over ranks."""
        if ws == 1:
            return list(times), list(counts)
        t = torch.tensor(times, dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        c = torch.tensor(counts, dtype=torch.int64, device=dev)
        torch.distributed.all_reduce(c)
        return t.tolist(), [int(x) for x in c.tolist()]

    def run_workload(name, steps, warmup, tune=True):
        views = build_views(name, runtime.find_formula, ws, rank, runtime.formula_names())
        nrays = workloads.rays(views)
        gbuf = runtime.GBuffer.allocate(nrays, device=dev)
        tr = ctx.autotune(views, gbuf) if tune else None
        opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, blocks_per_sm=tr.blocks_per_sm if tr else 0,
                                 refill_threshold=tr.refill_threshold if tr else 6, block=tr.block if tr else 0)
        graph = ctx.capture(views, gbuf, opts, stream=sptr)
        ms_p = timed(lambda: graph.launch(sptr), steps, warmup)
        st = ctx.stats()
        # the march kernel's and the shade pass's own device times: CUDA events the
        # library records around them on the launching stream (forward calls, L2 flushed)
        kt = []
        for i in range(warmup + steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            ctx.forward(views, gbuf, opts, stream=sptr)
            s2 = ctx.stats()
            if i >= warmup:
                kt.append((s2.march_ms, s2.shade_ms))
        kms = (sum(k[0] for k in kt) / len(kt), sum(k[1] for k in kt) / len(kt))
        plain_opts = runtime.make_opts(kernel=abi.ND_KERNEL_PLAIN)
        ms_plain = timed(lambda: ctx.forward(views, gbuf, plain_opts, stream=sptr), max(2, steps // 2), 1)
        # restore the persistent kernel's G-buffer for the error check
        graph.launch(sptr)
        stream.synchronize()
        graph.close()
        return views, nrays, gbuf, opts, tr, ms_p, ms_plain, st, kms

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    views, nrays, gbuf, opts, tune, ms_batched, ms_plain, st, kms = run_workload(args.workload, args.steps,
                                                                                  args.warmup)
    # end to end through the public call, as a renderer streams frames: every step
    # copies its view descriptors up (inside nd_march_forward) and reads its G-buffer
    # back into pinned host memory; with two G-buffers the read-back of step i (on a
    # copy stream) overlaps the march of step i + 1.  L2 flushed before every step.
    # The read-back is the reference's own G-buffer formats (fr:73-76): depth R32F,
    # normal RGBA16F (w = hit), plus the orbit trap and the step count.
    keys = ("depth", "normal_half", "trap", "steps")
    gbufs = []
    for _ in range(2):
        gb = runtime.GBuffer.allocate(nrays, device=dev)
        gb.normal = None
        gb.normal_half = torch.empty((nrays, 4), dtype=torch.float16, device=dev)
        gbufs.append(gb)
    hosts = [{k: torch.empty(getattr(gbufs[0], k).shape, dtype=getattr(gbufs[0], k).dtype, pin_memory=True)
              for k in keys} for _ in range(2)]
    d2h = sum(t.numel() * t.element_size() for t in hosts[0].values())
    h2d = len(views) * runtime.load_library().nd_sizeof(b"DevView")  # the view table nd_march_forward copies
    _, (d2h, h2d) = over_ranks([], [d2h, h2d])  # the whole job's copies per step
    copy_stream = torch.cuda.Stream(device=dev)

    def e2e_run(steps):
        done = [None, None]
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for i in range(steps):
            k = i % 2
            if done[k] is not None:
                stream.wait_event(done[k])  # the buffer's previous read-back has finished
            with torch.cuda.stream(stream):
                flush.fill_(1)
            ctx.forward(views, gbufs[k], opts, stream=sptr)
            marched = torch.cuda.Event()
            marched.record(stream)
            copy_stream.wait_event(marched)
            with torch.cuda.stream(copy_stream):
                for key, t in hosts[k].items():
                    t.copy_(getattr(gbufs[k], key), non_blocking=True)
                done[k] = torch.cuda.Event()
                done[k].record(copy_stream)
        stream.wait_stream(copy_stream)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / steps

    e2e_run(2)
    if ws > 1:
        torch.distributed.barrier()
    # a stream of frames: the last frame's read-back, which no march follows, stays
    # inside the timed region, spread over at least 20 frames
    e2e_steps = max(20, args.steps)
    ms_e2e = e2e_run(e2e_steps)
    extra = None
    if not args.no_extra and args.workload != "mandelbox_1080p":
        v2, n2, g2, _, tr2, ms2, ms2_plain, st2, _ = run_workload("mandelbox_1080p", max(2, args.steps // 2), 2)
        (ms2, ms2_plain), (n2_all, de2_all) = over_ranks([ms2, ms2_plain], [n2, st2.de_evals])
        extra = {"workload": "mandelbox_1080p (1920x1080 x 4 spp, shadow rays)", "rays_per_step": n2_all,
                 "value": n2_all / (ms2 * 1e-3) / 1e6, "unit": "Mrays/s", "ms_per_step": ms2,
                 "de_evals_per_s": de2_all / (ms2 * 1e-3),
                 "plain": n2_all / (ms2_plain * 1e-3) / 1e6, "batched_over_plain": ms2_plain / ms2,
                 "tune": {"kernel": tr2.kernel, "block": tr2.block, "blocks_per_sm": tr2.blocks_per_sm,
                          "refill_threshold": tr2.refill_threshold}}
        if rank == 0 and not args.no_cpu:
            torch.cuda.synchronize()
            extra["error_vs_fp64"] = sampled_errors(v2, g2, 32768, 9)
        del g2
    diff = other = None
    if not args.no_extra and ws == 1:
        diff = differentiation_step(ctx, stream, sptr, timed, max(2, args.steps // 2))
        other = small_and_deepzoom(ctx, sptr, timed, max(2, args.steps // 2), with_errors=not args.no_cpu)
    measured_fp32 = None
    if rank == 0:
        try:
            measured_fp32 = ctx.measure_fp32_peak(20.0)
        except runtime.NDError:
            measured_fp32 = None
    clk = clocks.stop()
    gnp = gbuf.numpy() if rank == 0 else None

    # rays: the sum over ranks (each marched its share of the one batch); times: the max
    (ms_batched, ms_plain, ms_e2e), (rays_total, de_all) = over_ranks([ms_batched, ms_plain, ms_e2e],
                                                                      [nrays, st.de_evals])
    if rank == 0:
        from numericdream_b200 import opcount

        flops_per_eval, per = opcount.flops_per_eval_for(views)
        flops = st.march_evals * flops_per_eval  # the march kernel's evaluations
        nominal = opcount.fp32_peak_tflops(clk.get("sm_mhz") or clk.get("sm_max_mhz"))
        peak = measured_fp32 if measured_fp32 else nominal
        achieved = flops / (kms[0] * 1e-3) / 1e12
        cpu, err = None, None
        if not args.no_cpu:
            c = run_cpu(views, seconds_budget=10.0, with_fp64=True)
            err = error_stats(views, gnp, c)
            ref = reference_lib()
            if ref:
                r = run_cpu_reference(ref, views, seconds_budget=10.0)
                cpu = {"value": r["rays_per_s"] / 1e6, "unit": "Mrays/s", "cores": r["cores"], "kind": "reference",
                       "sample": f"{r['rays']} rays in seeded runs of 64 consecutive rays over all 64 views "
                                 f"({r['seconds']:.1f} s, the reference's own march_to + estimate_normal "
                                 f"compiled for the host, FP32)",
                       "de_evals_per_s": r["evals_per_s"],
                       "port": {"value": c["rays_per_s"] / 1e6, "de_evals_per_s": c["evals_per_s"],
                                "kind": "the oracle's FP32 march"}}
            else:
                cpu = {"value": c["rays_per_s"] / 1e6, "unit": "Mrays/s", "cores": c["cores"], "kind": "port",
                       "sample": f"{c['rays']} rays in seeded runs of 64 consecutive rays over all 64 views "
                                 f"({c['seconds']:.1f} s, FP32 oracle march)",
                       "de_evals_per_s": c["evals_per_s"]}
        line = {
            "metric": METRIC, "value": rays_total / (ms_batched * 1e-3) / 1e6, "unit": "Mrays/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_batched, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded views, no dataset)",
            "config": config_of(args.workload, views, ws, rays_total),
            "de_evals_per_s": de_all / (ms_batched * 1e-3),
            "plain": {"value": rays_total / (ms_plain * 1e-3) / 1e6, "unit": "Mrays/s", "ms_per_step": ms_plain,
                      "kind": "one plain launch per view, one thread per ray"},
            "batched_over_plain": ms_plain / ms_batched,
            "e2e": {"value": rays_total / (ms_e2e * 1e-3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e, "steps": e2e_steps,
                    "kind": "nd_march_forward from host view descriptors, G-buffer (depth R32F, normal RGBA16F, "
                            "trap, steps: 20 B per ray) read back to pinned host memory every step; two G-buffers, "
                            "read-back of step i overlapping the march of step i+1; the last read-back inside "
                            "the timed region"},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "traffic": NCU_TRAFFIC.get(args.workload, {}).get("march"),
                         "traffic_forward": sum(NCU_TRAFFIC.get(args.workload, {}).values()) or None,
                         "traffic_note": "DRAM bytes per launch of the march (traffic) and of the whole forward, "
                                         "march + surface pass (traffic_forward), from one ncu capture",
                         "issue_active": NCU_ISSUE.get(args.workload),
                         "issue_note": "the march's share of issue slots busy (ncu smsp__issue_active, one "
                                       "capture): the bound of this scalar, branchy code, whose FP32 "
                                       "add/mul/fma are under half of the instructions it issues",
                         "kernel": "persistent_kernel (march); FLOPs = its DE evaluations x FLOPs per "
                                   "evaluation, over its CUDA-event time",
                         "kernel_ms": kms[0], "shade_pass_ms": kms[1],
                         "flops_per_eval": flops_per_eval, "sfu_per_eval": per["sfu"],
                         "peak_source": ("measured: nd_measure_fp32_peak, independent FFMA chains on this GPU "
                                         "(CUDA events); FP32 is not in MEASURED_PEAKS.json")
                         if measured_fp32 else "nominal: 148 SMs x 128 FP32 lanes x 2 x sampled SM clock",
                         "peak_nominal": nominal},
            "error_vs_fp64": err, "cpu_baseline": cpu, "clocks": clk,
            # per replayed forward: the counter clear, the march, the surface pass, and
            # the shadow pass when a view casts shadow rays
            "gpu_launches": (3 + (1 if any(v.shadow for v in views) else 0)) * args.steps,
            "stats": {"de_evals": st.de_evals, "march": st.march_evals, "normal": st.normal_evals,
                      "shadow": st.shadow_evals, "trap": st.trap_evals, "hits": st.hits, "refills": st.refills},
            "tune": {"kernel": tune.kernel, "block": tune.block, "blocks_per_sm": tune.blocks_per_sm,
                     "refill_threshold": tune.refill_threshold} if tune else None,
            "second_workload": extra,
            "differentiation": diff,
            "other_configs": other,
        }
        print(json.dumps(line))
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
