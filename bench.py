"""Benchmark of the B200 sphere-tracing pass.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one forward march over the whole workload.  The default workload is the
batched one (64 views of mixed formulas and uneven sizes in one persistent launch,
replayed as a CUDA graph); the plain per-view launch of the same views is timed
beside it.  Rank 0 prints one JSON line.

value      rays/s of the batched persistent kernel, device time (CUDA events on the
           launching stream), inputs resident; L2 is flushed between steps.
e2e        the same metric through the public C ABI call with host view descriptors
           and the G-buffer read back to pinned host memory every step.
roofline   FP32-pipe roofline of the march kernel: algorithmic FLOPs per launch
           (DE evaluations x FLOPs per evaluation of each formula, counted by the
           op-counting instantiation of the same formula code) / kernel time.
cpu_baseline  the oracle's FP32 march (same formulas, same march) on all host
           cores over a bounded sample of the workload's rays.

--impl reference times the CPU implementation of the path (the oracle's FP32
march, every host thread) on the same workload and metric: the reference app
itself only runs through WebGPU, which this machine cannot run.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Mrays/s & DE-evals/s on 1 B200, batched vs plain, at stated FP64 error"


def _dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

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
        return self.summary()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            try:
                sm.append(float(s[1]))
                mx = float(s[2])
            except (ValueError, IndexError):
                continue
            for i, n in enumerate(names):
                if len(s) > 5 + i and s[5 + i].lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_views(name, resolve):
    from numericdream_b200 import workloads

    if name == "batched_64":
        return workloads.batched_64(resolve)
    if name == "mandelbox_1080p":
        return workloads.mandelbox_1080p(resolve)
    if name == "mandelbulb_256":
        return workloads.mandelbulb_256(resolve)
    raise SystemExit(f"unknown workload {name}")


def config_of(name, views):
    from numericdream_b200 import workloads

    return {"workload": name, "views": len(views), "rays_per_step": workloads.rays(views),
            "max_steps": int(views[0].max_steps), "de": "fp32", "t": "fp64",
            "l2": "flushed between steps (256 MiB write)"}


def cpu_sample(views, target_rays, seed=0):
    """A bounded, seeded, evenly spread subset of (view, first ray, count) chunks."""
    import random

    from numericdream_b200 import abi

    rng = random.Random(seed)
    total = sum(abi.rays_of(v) for v in views)
    frac = min(1.0, target_rays / max(total, 1))
    chunks = []
    for v in views:
        n = abi.rays_of(v)
        k = max(1, int(n * frac))
        # contiguous runs of 64 rays spread over the view
        runs = max(1, k // 64)
        for _ in range(runs):
            first = rng.randrange(0, max(1, n - 64))
            chunks.append((v, first, min(64, n - first)))
    return chunks


def run_cpu(views, seconds_budget=15.0, nthreads=0):
    """Time the oracle's FP32 march on all host cores over a bounded sample."""
    from numericdream_b200 import runtime
    from oracle import pyoracle

    cores = nthreads or pyoracle.max_threads()
    probe = cpu_sample(views, 2048, seed=1)
    t0 = time.perf_counter()
    nr = 0
    for v, first, n in probe:
        pyoracle.render(v, runtime.formula_name(v.formula), precision=32, nthreads=cores, first=first, n=n)
        nr += n
    dt = max(time.perf_counter() - t0, 1e-6)
    target = int(nr / dt * seconds_budget)
    chunks = cpu_sample(views, max(target, 4096), seed=2)
    t0 = time.perf_counter()
    rays = 0
    evals = 0
    for v, first, n in chunks:
        o = pyoracle.render(v, runtime.formula_name(v.formula), precision=32, nthreads=cores, first=first, n=n)
        rays += n
        evals += int(o["evals"].astype("int64").sum())
    dt = time.perf_counter() - t0
    return {"rays_per_s": rays / dt, "evals_per_s": evals / dt, "rays": rays, "seconds": dt, "cores": cores}


def reference_arm(args):
    ws, rank, _ = _dist_env()
    if rank != 0:
        return 0
    from numericdream_b200 import runtime

    try:
        runtime.load_library()
        resolve = runtime.find_formula
    except ImportError as e:
        print(json.dumps({"impl": "reference", "unavailable": f"formula table not built: {e}"}))
        return 0
    views = build_views(args.workload, resolve)
    per = []
    res = None
    for i in range(args.warmup + args.steps):
        res = run_cpu(views, seconds_budget=max(2.0, 60.0 / max(args.steps + args.warmup, 1)))
        if i >= args.warmup:
            per.append(res)
    v = sum(r["rays_per_s"] for r in per) / len(per) / 1e6
    line = {"metric": METRIC, "value": v, "unit": "Mrays/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_of(args.workload, views),
            "de_evals_per_s": sum(r["evals_per_s"] for r in per) / len(per),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": res["cores"], "kind": "port",
                             "sample": f"{res['rays']} rays per step, seeded runs of 64 rays spread over all views"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CPU FP32 restatement of the reference march (the reference runs only through WebGPU)"}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched_64")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    import numpy as np
    import torch

    from numericdream_b200 import abi, runtime, workloads

    ws, rank, local = _dist_env()
    if ws > 1:
        import torch.distributed as dist
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    ctx = runtime.Context(local)
    views = build_views(args.workload, runtime.find_formula)
    nrays = workloads.rays(views)
    gbuf = runtime.GBuffer.allocate(nrays, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    tune = None
    if not args.no_autotune:
        tune = ctx.autotune(views, gbuf)
    opts = runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, blocks_per_sm=tune.blocks_per_sm if tune else 0,
                             refill_threshold=tune.refill_threshold if tune else 8)
    graph = ctx.capture(views, gbuf, opts, stream=sptr)

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

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    ms_batched = timed(lambda: graph.launch(sptr), args.steps, args.warmup)
    st = ctx.stats()
    de_evals = st.de_evals
    plain_opts = runtime.make_opts(kernel=abi.ND_KERNEL_PLAIN)
    ms_plain = timed(lambda: ctx.forward(views, gbuf, plain_opts, stream=sptr), max(2, args.steps // 2), 1)
    # end to end through the public call: host descriptors in, G-buffer to pinned host
    host = {k: torch.empty(getattr(gbuf, k).shape, dtype=getattr(gbuf, k).dtype, pin_memory=True)
            for k in ("depth", "normal", "trap", "steps")}
    d2h = sum(t.numel() * t.element_size() for t in host.values())
    h2d = len(views) * 512

    def e2e_step():
        ctx.forward(views, gbuf, opts, stream=sptr)
        for k, t in host.items():
            t.copy_(getattr(gbuf, k), non_blocking=True)

    ms_e2e = timed(e2e_step, max(2, args.steps // 2), 1)
    clk = clocks.stop()

    if ws > 1:
        t = torch.tensor([ms_batched, ms_plain, ms_e2e], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_batched, ms_plain, ms_e2e = t.tolist()
    graph.close()
    rays_total = nrays * ws
    value = rays_total / (ms_batched * 1e-3) / 1e6
    line = None
    if rank == 0:
        from numericdream_b200 import opcount

        flops_per_eval, fcount = opcount.flops_per_eval_for(views)
        flops = de_evals * flops_per_eval
        peak = opcount.fp32_peak_tflops(clk.get("sm_max_mhz"))
        achieved = flops / (ms_batched * 1e-3) / 1e12
        cpu = None
        if not args.no_cpu:
            c = run_cpu(views, seconds_budget=15.0)
            cpu = {"value": c["rays_per_s"] / 1e6, "unit": "Mrays/s", "cores": c["cores"], "kind": "port",
                   "sample": f"{c['rays']} rays in seeded runs of 64 spread over all views ({c['seconds']:.1f} s)"}
        line = {
            "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_batched, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_of(args.workload, views),
            "de_evals_per_s": de_evals * ws / (ms_batched * 1e-3),
            "plain": {"value": rays_total / (ms_plain * 1e-3) / 1e6, "unit": "Mrays/s", "ms_per_step": ms_plain},
            "batched_over_plain": ms_plain / ms_batched,
            "e2e": {"value": rays_total / (ms_e2e * 1e-3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None, "flops_per_eval": flops_per_eval,
                         "peak_source": "nominal SMs x 128 FP32 lanes x 2 x max SM clock"},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": args.steps,
            "tune": {"kernel": tune.kernel, "blocks_per_sm": tune.blocks_per_sm,
                     "refill_threshold": tune.refill_threshold} if tune else None,
        }
        print(json.dumps(line))
    ctx.close()
    if ws > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
