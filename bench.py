"""Benchmark of the FRW hot path on B200: walks/s (and time to 0.1% rel. SE).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (one "step"): 1e7 floating random walks from conductor 0 of a
10,000-rectangle layout on [0,1e4]^2 (integer corners, sizes 5-50, L-inf gap
>= 2, seed 0xF4A7+2), Gaussian surface = target grown by 1 unit, uniform start,
capacitance row accumulated.  Synthetic data: the reference ships no benchmark
suite.  Under torchrun every rank runs its own 1e7 walks (Philox stream =
rank; weak scaling) and the per-conductor rows are summed with one NCCL
all-reduce inside the step.

`value`  : walks/s with the layout resident in HBM (device events, max over ranks).
`e2e`    : walks/s through the public C ABI from pinned host rects: layout
           upload + tree build + walks + result rows back, every step.
`--impl reference`: the reference's own CPU walk (RandomWalk as shipped,
           compiled from its sources into oracle/_ref) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import re
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "engineer-thesis_b200"))

WORKLOAD = dict(workload="frw-c2-10k-rects-1e7-walks", rects=10_000, domain=1e4, walks=10_000_000,
                target=0, gauss="offset-1", start="uniform", layout_seed=0xF4A7 + 2)
METRIC = "walks/s (plain FRW, 10k-rect layout, 1e7 walks/step, capacitance row)"


def algorithmic_bytes_per_query(n_rects: int) -> int:
    """16 B per node on the location path (D levels) + 16 rects of 16 B."""
    d = math.ceil(math.log(max(n_rects / 4, 1), 4)) + 1
    return 16 * d + 16 * 16


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(walks_per_launch: int):
    """DRAM bytes of one walk-kernel launch of `walks_per_launch` walks, scaled
    from the committed ncu capture (a smaller launch of the same kernel and
    layout; the traffic is accumulator flushes, proportional to walks)."""
    p = os.path.join(ROOT, "profiles", "walk_kernel_c2.md")
    if not os.path.exists(p):
        return None
    txt = open(p).read()
    m = re.search(r"dram_bytes_per_launch\s*=\s*([0-9.eE+]+)", txt)
    w = re.search(r"walks_per_launch\s*=\s*([0-9.eE+]+)", txt)
    if not (m and w):
        return None
    return float(m.group(1)) * walks_per_launch / float(w.group(1))


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        rows = [r.split(", ") for r in self.out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "samples": len(rows),
                "reasons": reasons}


# ------------------------------------------------------------ reference arm
def _ref_worker(args):
    rects, bounds, target, seconds, wid = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    R = O.Ref(rects=rects, bounds=bounds)
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        R.walks_as_shipped(target, 4)
        done += 4
    return done, time.perf_counter() - t0


def reference_rate(rects, bounds, target, seconds, cores):
    """Walks/s of the shipped reference CPU walk on `cores` processes."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        res = pool.map(_ref_worker, [(rects, bounds, target, seconds, i) for i in range(cores)])
    return sum(d for d, _ in res) / max(t for _, t in res), sum(d for d, _ in res)


def reference_available():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "librefcpu.so"))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import frw

    rects = frw.generate_layout(WORKLOAD["layout_seed"], WORKLOAD["rects"], WORKLOAD["domain"]).astype(np.float64)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    bounds = O.layer_bounds(rects)
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/librefcpu.so not built "
                          "(needs the reference sources at build time)"}))
        return 0
    cores = os.cpu_count() or 1
    step_s = 2.0
    for _ in range(args.warmup):
        reference_rate(rects, bounds, WORKLOAD["target"], 0.5, cores)
    t0 = time.perf_counter()
    total = 0
    for _ in range(args.steps):
        _, n = reference_rate(rects, bounds, WORKLOAD["target"], step_s, cores)
        total += n
    el = time.perf_counter() - t0
    v = total / el
    cfg = dict(WORKLOAD, gauss="reference scale 1.5", start="reference Green CDF", walks=f"~{step_s}s sample/step")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "walks/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": cfg,
        "cpu_baseline": {"value": v, "unit": "walks/s", "cores": cores, "kind": "reference",
                         "sample": f"RandomWalk as shipped (per-walk rng_init), {args.steps} x {step_s}s on "
                                   f"{cores} processes, {total} walks"},
        "e2e": {"value": v, "unit": "walks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


# ------------------------------------------------------------------ our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="frw", choices=["frw", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--walks", type=int, default=None, help="override walks per step (profiling runs)")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    if args.walks:
        WORKLOAD["walks"] = args.walks
    if args.impl == "reference":
        return run_reference(args)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    import frw
    from frw import shard

    W = WORKLOAD
    rects = frw.generate_layout(W["layout_seed"], W["rects"], W["domain"])
    # CPU baseline first (spawned pool, before heavy GPU work), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and reference_available():
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        cores = os.cpu_count() or 1
        rate, n = reference_rate(rects.astype(np.float64), O.layer_bounds(rects.astype(np.float64)), W["target"],
                                 args.cpu_seconds, cores)
        cpu = {"value": rate, "unit": "walks/s", "cores": cores, "kind": "reference",
               "sample": f"reference RandomWalk as shipped (per-walk rng_init, reference scale-1.5 surface and "
                         f"Green-CDF start) on the same layout and target, {args.cpu_seconds:.0f}s on {cores} "
                         f"processes, {n} walks"}

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    o = frw.capacitance_opts(1.0, stream_id=shard.plan(W["walks"], rank)["stream"])
    L = frw.Layout.from_rects(rects, device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def step(seed):
        r = L.walk(W["target"], W["walks"], seed, o, stream=stream.cuda_stream)
        if dist is not None:  # the one exchange: sum of the packed rows (NCCL)
            shard.all_reduce_rows(torch.as_tensor(shard.result_rows(r, L.n), device=dev))
        return r

    for i in range(args.warmup):
        step(1000 + i)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kern_ms, hops, results = [], 0, []
    with Clocks(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            r = step(i)
            ev[i][1].record(stream)
            kern_ms.append(r.kernel_ms)
            hops += r.hops_total
            results.append(r)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    if dist is not None:
        t = torch.tensor([t_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    walks_total = W["walks"] * args.steps * world
    value = walks_total / (t_ms * 1e-3)

    # e2e through the public ABI from pinned host memory
    pinned = torch.from_numpy(rects).pin_memory()
    ptr = pinned.data_ptr()
    import ctypes

    def e2e_step(seed):
        h = ctypes.c_void_p()
        frw._check(frw.lib().frw_layout_create(ctypes.cast(ptr, frw._F), W["rects"], None, local,
                                               ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        Le = frw.Layout(h, W["rects"])
        r = Le.walk(W["target"], W["walks"], seed, o, stream=stream.cuda_stream)
        Le.close()
        return r

    e2e_ms, nrows = float("nan"), 0
    if not args.no_e2e:
        e2e_step(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_steps = max(3, args.steps // 2)
        e0.record(stream)
        for i in range(e2e_steps):
            nrows = len(e2e_step(50 + i).conductor)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / e2e_steps

    if rank == 0:
        last = results[-1]
        i0 = int(np.searchsorted(last.conductor, W["target"]))
        rel_se = float(last.cap_se[i0] / abs(last.cap[i0]))
        hbar = hops / (W["walks"] * args.steps)
        bq = algorithmic_bytes_per_query(W["rects"])
        kms = statistics.median(kern_ms)
        achieved = W["walks"] * hbar * bq / (kms * 1e-3) / 1e9
        peak, peak_kind = measured_peak_hbm()
        traffic = profiled_traffic(W["walks"])
        out = {
            "metric": METRIC, "value": value, "unit": "walks/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(W, l2="flushed between steps (256 MiB write)", parallelism=f"walks x{world}",
                           time_to_rel_se_1e3_s=t_ms / args.steps * 1e-3 * (rel_se / 1e-3) ** 2,
                           c00_rel_se_per_step=rel_se, mean_hops=hbar),
            "e2e": {"value": W["walks"] / (e2e_ms * 1e-3), "unit": "walks/s",
                    "h2d_bytes_per_step": W["rects"] * 16 + 32,
                    "d2h_bytes_per_step": nrows * 32 + 64},
            "gpu_launches": 3 * args.steps,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "note": f"walk kernel; algorithmic {bq} B/query x {hbar:.2f} queries/walk; peak {peak_kind} "
                                 "(the tree is L2-resident, so HBM is an upper-bound denominator)"},
            "clocks": clk.summary(),
        }
        if cpu:
            out["cpu_baseline"] = cpu
        print(json.dumps(out))
    L.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
