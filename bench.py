"""Benchmark of the FRW hot path on B200: walks/s (and time to 0.1% rel. SE).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload of one step (`config`, the same in both arms): 1e8 floating random
walks from conductor 0 of a 10^6-rectangle layout on [0,1e5]^2 (integer
corners, sizes 5-50, L-inf gap >= 2, seed 0xF4A7+3), with the reference's own
walk definition: Gaussian surface = the target scaled by 1.5 and bisected
until it clears its neighbours (creatGaussianSurfFrom), start point = a
Green-CDF bin mapped on that surface (RandomWalk), estimator = per-conductor
end counts (getAvgPathLen).  Synthetic data: the reference ships no benchmark
suite.  Under torchrun every rank runs its own 1e8 walks (Philox stream =
rank; weak scaling) and the per-conductor rows are summed once per step: each
rank's nonzero rows only (frw_rows_compact), one NCCL all-gather.

`value`  : walks/s with the layout resident in HBM and the rows left on the
           device (frw_walk_device; device events, max over ranks).
`e2e`    : walks/s through the C ABI from pinned host rects: layout upload +
           tree and cell-list build + walks + result rows back, every step.
`--impl reference`: the reference's own CPU walk (RandomWalk as shipped,
           compiled from its sources into oracle/_ref) on all host cores, on
           the same layout (made by the oracle's generator: no product code
           is loaded in that process) and the same walk definition.
Sub-lines: `c2` (10^4 rects, capacitance row, offset-1 surface), `c3_capacitance`
(10^6 rects, capacitance row), `collision_queries`, `time_to_0.1pct_rel_se`
(plain vs control variate on 10^6 rects), `batched` (256 layouts) and
`walk3d` (the 3-D walk over box conductors).
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

WORKLOAD = dict(workload="frw-c3-1e6-rects-1e8-walks", rects=1_000_000, domain=1e5, walks=100_000_000, target=0,
                gauss="target scaled by 1.5, bisected to clear its neighbours (reference creatGaussianSurfFrom)",
                start="Green-CDF bin on the Gaussian perimeter (reference RandomWalk)",
                estimator="per-conductor end counts, fraction ending elsewhere (reference getAvgPathLen)",
                layout_seed=0xF4A7 + 3,
                l2="working set above the 126 MB L2 (cell lists 0.8 GB); the GPU arm also writes 256 MiB "
                   "between steps")
METRIC = "walks/s (plain FRW, 10^6-rect layout, 1e8 walks/step, reference surface, start and estimator)"
PROFILE = os.path.join(ROOT, "profiles", "walk_kernel_c3.md")
PROFILE3 = os.path.join(ROOT, "profiles", "walk3d_kernel_1e4_boxes.md")


def algorithmic_bytes_per_query(n_rects: int) -> int:
    """16 B per node on the location path (D levels) + 16 rects of 16 B."""
    d = math.ceil(math.log(max(n_rects / 4, 1), 4)) + 1
    return 16 * d + 16 * 16


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_figures(path=PROFILE):
    """key = value lines of a committed ncu summary (numbers only)."""
    if not os.path.exists(path):
        return {}
    out = {}
    for m in re.finditer(r"^\s*([a-z0-9_]+)\s*=\s*([0-9.eE+-]+)\s*$", open(path).read(), re.M):
        out[m.group(1)] = float(m.group(2))
    return out


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


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


# ------------------------------------------------------------ CPU legs
# Worker processes build their layout index once, in the pool initialiser
# (outside every timed call), from the oracle's generator -- the product
# library is never loaded in them.
_W = {}


def _cpu_init(kind, seed, n, domain, target):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    rects = O.generate_layout(seed, n, domain)
    bounds = O.layer_bounds(rects)
    _W.update(kind=kind, target=target, O=O)
    if kind == "reference":
        _W["R"] = O.Ref(rects=rects, bounds=bounds)
    else:
        G = O.Grid(rects, bounds)
        _W["G"] = G
        if kind == "port":  # the benchmark's own walk definition (reference surface and start)
            _W["cfg"] = G.walk_cfg(target=target, gauss_mode=O.GAUSS_SCALE, gauss_param=1.5,
                                   start_mode=O.START_GREEN, seed=7, stream=os.getpid() & 0xFFFF)
        else:  # "port_capacitance": offset-1 surface, uniform start, capacitance weights
            _W["cfg"] = G.walk_cfg(target=target, gauss_mode=O.GAUSS_OFFSET, gauss_param=1.0,
                                   start_mode=O.START_UNIFORM, seed=7, stream=os.getpid() & 0xFFFF)
        _W["next"] = 0


def _cpu_run(args):
    seconds, wid, mode = args
    done, k, t0 = 0, 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        if _W["kind"] == "reference":
            if mode == "shipped":  # RandomWalk itself: per-walk rng_init, as shipped
                _W["R"].walks_as_shipped(_W["target"], 4)
                done += 4
            else:  # the same walk loop with JKISS seeded once per 64 walks
                _W["R"].walks_seeded(_W["target"], 64, seed=(wid + 1, k + 7, 0x5EED, 0xC0FFEE))
                done += 64
        else:
            _W["G"].walks(_W["cfg"], _W["next"], 1024)
            _W["next"] += 1024
            done += 1024
        k += 1
    return done


class CpuLeg:
    """`cores` single-threaded worker processes on one layout."""

    def __init__(self, kind, cores, seed, n, domain, target):
        self.cores = cores
        self.pool = mp.get_context("spawn").Pool(cores, initializer=_cpu_init,
                                                 initargs=(kind, seed, n, domain, target))
        self.run(0.05, "seeded")  # every worker has built its index

    def run(self, seconds, mode="shipped"):
        """(walks/s over the call's wall time, walks)."""
        t0 = time.perf_counter()
        done = sum(self.pool.map(_cpu_run, [(seconds, i, mode) for i in range(self.cores)], chunksize=1))
        return done / (time.perf_counter() - t0), done

    def close(self):
        self.pool.terminate()
        self.pool.join()


def reference_available():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "librefcpu.so"))


def run_reference(args):
    """The reference arm: RandomWalk as shipped on every host core, on the
    benchmark's layout and walk definition; each step a bounded sample."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/librefcpu.so not built "
                          "(needs the reference sources at build time)"}))
        return 0
    W = WORKLOAD
    cores = host_cores()
    step_s = 2.0
    leg = CpuLeg("reference", cores, W["layout_seed"], W["rects"], W["domain"], W["target"])
    for _ in range(args.warmup):
        leg.run(0.5)
    total, wall = 0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, n = leg.run(step_s)
        wall += time.perf_counter() - t0
        total += n
    leg.close()
    v = total / wall
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "walks/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(W),
        "cpu_baseline": {"value": v, "unit": "walks/s", "cores": cores, "kind": "reference",
                         "sample": f"RandomWalk as shipped (per-walk rng_init), {args.steps} x {step_s}s of walks on "
                                   f"{cores} processes, {total} walks; layout from the oracle's generator, "
                                   "reference CPU quadtree built once per process outside the timing"},
        "e2e": {"value": v, "unit": "walks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def cpu_baselines(seconds):
    """Rank 0 at N = 1, before any GPU work: the reference as shipped, its walk
    loop seeded once, and the FP64 restatement, all on the headline layout."""
    W = WORKLOAD
    cores = host_cores()
    out = {}
    if reference_available():
        leg = CpuLeg("reference", cores, W["layout_seed"], W["rects"], W["domain"], W["target"])
        rate, n = leg.run(seconds)
        rate1, n1 = leg.run(seconds / 2, "seeded")
        leg.close()
        out = {"value": rate, "unit": "walks/s", "cores": cores, "kind": "reference", "per_core": rate / cores,
               "sample": f"reference RandomWalk as shipped (per-walk rng_init, its CPU quadtree) on the headline "
                         f"layout and walk definition, {seconds:.0f}s on {cores} processes, {n} walks",
               "seeded_once": {"value": rate1, "per_core": rate1 / cores,
                               "sample": f"the same reference walk loop with JKISS seeded once per 64 walks, "
                                         f"{seconds / 2:.0f}s on {cores} processes, {n1} walks"}}
    leg = CpuLeg("port", cores, W["layout_seed"], W["rects"], W["domain"], W["target"])
    rate2, n2 = leg.run(seconds / 4)
    leg.close()
    port = {"value": rate2, "unit": "walks/s", "cores": cores, "kind": "port", "per_core": rate2 / cores,
            "sample": f"the FP64 CPU restatement (oracle/, complete queries on a uniform grid index) on the "
                      f"headline layout and walk definition, {seconds / 4:.1f}s on {cores} processes, {n2} walks"}
    if out:
        out["port"] = port
        return out
    return port


# ------------------------------------------------------------ headline runs
HEADLINE = dict(workload="frw-c5-1e6-rects", rects=1_000_000, domain=1e5, layout_seed=0xF4A7 + 3, target=0,
                start_grid=16384, cv_train_walks=1_000_000, cv_epochs=4, rel_se=1e-3)


def time_to_rel_se(frw, device, stream):
    """Wall time to reach 0.1% rel. SE of C_00 on the 10^6-rect layout, plain vs
    control variate (training included), each run as: pilot batch -> walks needed
    -> main batch.  Device time from CUDA events, wall time from the host clock."""
    import torch

    H = HEADLINE
    rects = frw.generate_layout(H["layout_seed"], H["rects"], H["domain"])
    L = frw.Layout.from_rects(rects, device=device)
    o = frw.capacitance_opts(1.0, start_grid=H["start_grid"])
    # untimed warm-up of both paths (module loading, memory-pool growth)
    L.walk(0, 1_000_000, seed=1, o=o)
    w = frw.ControlVariate(L, H["target"], o, frw.cv_opts(train_walks=H["cv_train_walks"], epochs=1))
    w.walk(1_000_000, seed=2)
    w.close()
    torch.cuda.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) * 1e-3, time.perf_counter() - t0

    def plain():
        pilot = L.walk(H["target"], 2_000_000, seed=11, o=o)
        c, se = pilot.row(H["target"])[1:]
        need = int(pilot.walks * (se / abs(c) / H["rel_se"]) ** 2 * 1.05) + 1
        main_ = L.walk(H["target"], need, seed=12, o=o)
        n = pilot.walks + main_.walks
        i0, i1 = (np.searchsorted(r.conductor, H["target"]) for r in (pilot, main_))
        s1 = pilot.sum_w[i0] + main_.sum_w[i1]
        s2 = pilot.sum_w2[i0] + main_.sum_w2[i1]
        mean = s1 / n
        se = np.sqrt(max(s2 / n - mean * mean, 0.0) * n / (n - 1) / n)
        return {"walks": n, "c00": mean, "rel_se": se / abs(mean)}

    def with_cv():
        cv = frw.ControlVariate(L, H["target"], o, frw.cv_opts(train_walks=H["cv_train_walks"],
                                                              epochs=H["cv_epochs"]))
        pilot = cv.walk(1_000_000, seed=21)
        need = int(pilot.walks * (pilot.cv_se / abs(pilot.cv) / H["rel_se"]) ** 2 * 1.05) + 1
        main_ = cv.walk(max(need, 2), seed=22)
        n = pilot.walks + main_.walks
        c = (pilot.cv * pilot.walks + main_.cv * main_.walks) / n
        se = np.sqrt((pilot.cv_se * pilot.walks) ** 2 + (main_.cv_se * main_.walks) ** 2) / n
        info = cv.info
        out = {"walks": n, "c00": c, "rel_se": se / abs(c), "variance_reduction": main_.variance_ratio,
               "train_walks": info.train_walks, "train_device_s": info.train_ms * 1e-3,
               "exact_mean_device_s": info.quad_ms * 1e-3, "exact_mean_points": info.quad_points}
        cv.close()
        return out

    p, p_dev, p_wall = timed(plain)
    c, c_dev, c_wall = timed(with_cv)
    L.close()
    return {"workload": H["workload"], "target_rel_se": H["rel_se"], "start_grid": H["start_grid"],
            "plain": dict(p, device_s=p_dev, wall_s=p_wall),
            "cv": dict(c, device_s=c_dev, wall_s=c_wall),
            "speedup_wall": p_wall / c_wall, "speedup_device": p_dev / c_dev,
            "cv_wall_s_training_amortised": c_wall - c["train_device_s"] - c["exact_mean_device_s"],
            "speedup_wall_training_amortised": p_wall / (c_wall - c["train_device_s"] - c["exact_mean_device_s"]),
            "agree_sigma": abs(p["c00"] - c["c00"]) / np.hypot(p["c00"] * p["rel_se"], c["c00"] * c["rel_se"])}


# ------------------------------------------------------------ queries
def query_rates(frw, L, device, stream, sets):
    """drawBiggestSquareAtPoint + checkCollisons(point) per point, batched on
    device buffers: (name, points, seed, repetitions) per set, points uniform
    in the layout's bounds."""
    import torch

    b = L.bounds
    out = {}
    for name, n, seed, reps in sets:
        rng = np.random.default_rng(seed)
        pts = np.stack([rng.uniform(b[0], b[2], n), rng.uniform(b[1], b[3], n)], 1)
        p = torch.as_tensor(pts, device=device)
        sq = torch.empty((n, 4), dtype=torch.float64, device=device)
        hit = torch.empty(n, dtype=torch.int64, device=device)
        L.query_device(p, sq, hit, stream.cuda_stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            L.query_device(p, sq, hit, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"points": n, "ms": ms, "queries_per_s": n / (ms * 1e-3)}
        del p, sq, hit
    return out


# ------------------------------------------------------------ sub-lines on the capacitance estimator
C2 = dict(workload="frw-c2-10k-rects-1e7-walks", rects=10_000, domain=1e4, walks=10_000_000, target=0,
          gauss="offset-1", start="uniform", estimator="capacitance row", layout_seed=0xF4A7 + 2)
C3CAP = dict(workload="frw-c3-1e6-rects-1e8-walks-capacitance", rects=1_000_000, domain=1e5, walks=100_000_000,
             target=0, gauss="offset-1", start="uniform", estimator="capacitance row", layout_seed=0xF4A7 + 3)


def device_rows_run(frw, W, o, device, stream, steps, flush):
    """walks/s of frw_walk_device on layout W (rows left on the device, L2
    flushed between steps), the C_00 row and the mean hop count."""
    import torch

    rects = frw.generate_layout(W["layout_seed"], W["rects"], W["domain"])
    L = frw.Layout.from_rects(rects, device=device)
    n = L.n
    dev = torch.device("cuda", device)
    rows_i = torch.zeros(n + 4, dtype=torch.int64, device=dev)
    rows_f = torch.zeros(2 * n, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)

    def step(seed):
        rows_i.zero_()
        rows_f.zero_()
        L.walk_device(W["target"], W["walks"], seed, o, rows_i[:n], rows_f[:n], rows_f[n:], rows_i[n:], status,
                      stream.cuda_stream)

    for i in range(3):
        step(900 + i)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        step(700 + i)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if int(status.item()) != 0:
        raise RuntimeError(f"walk kernel reported status {int(status.item()):#x}")
    ms = statistics.median(a.elapsed_time(b) for a, b in ev)
    ri, rf = rows_i.cpu().numpy(), rows_f.cpu().numpy()
    st = ri[n:]
    nw = float(W["walks"])
    m1 = rf[W["target"]] / nw
    var = max(rf[n + W["target"]] / nw - m1 * m1, 0.0) * nw / (nw - 1.0)
    hbar = float(st[2]) / float(st[3])
    bq = algorithmic_bytes_per_query(W["rects"])
    peak, kind = measured_peak_hbm()
    ach = W["walks"] * hbar * bq / (ms * 1e-3) / 1e9
    out = {"workload": W["workload"], "config": W, "kernel_ms": ms, "walks_per_s": W["walks"] / (ms * 1e-3),
           "mean_hops": hbar, "c00": m1, "c00_rel_se": float(np.sqrt(var / nw) / abs(m1)) if m1 else None,
           "conductors_reached": int((ri[:n] > 0).sum()),
           "roofline_frac": ach / peak, "roofline_note": f"{bq} B/query x {hbar:.2f} queries/walk of {kind} HBM"}
    L.close()
    return out


# ------------------------------------------------------------ 3-D path
W3D = dict(workload="frw3-1e4-boxes-1e7-walks", boxes=10_000, domain=2000.0, zdomain=400.0, edges="5-50 (z 5-20)",
           gap=2, walks=10_000_000, target=0, gauss_offset=1.0, nsample=50, layout_seed=0xF4A7 + 6)


def _port3_worker(args):
    boxes, target, seconds, wid = args
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    B = O.Boxes3(boxes, grid=True)
    cfg = B.cfg(target=target, offset=W3D["gauss_offset"], seed=11, stream=wid, nsample=W3D["nsample"])
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        B.walks(cfg, done, 512)
        done += 512
    return done, time.perf_counter() - t0


def walk3d_run(frw, device, stream, steps, cpu_seconds, cores, sm_mhz=None):
    """The 3-D walk (box conductors, cube transition domains from the
    reference's unit-cube Green's function): 10^4 boxes, 1e7 walks per step,
    capacitance row of box 0.  Per-walk records equal the FP64 oracle's
    (GPU tests); e2e includes the box upload and grid build every step."""
    import torch

    b = frw.generate_layout3(W3D["layout_seed"], W3D["boxes"], W3D["domain"], W3D["zdomain"], 5, 50, 5, 20,
                             W3D["gap"])
    o = frw.opts3(gauss_offset=W3D["gauss_offset"], nsample=W3D["nsample"])
    L = frw.Layout3.from_boxes(b, device=device)
    L.walk(W3D["target"], 1_000_000, 1, o, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = [L.walk(W3D["target"], W3D["walks"], 300 + k, o, stream=stream.cuda_stream) for k in range(steps)]
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    kms = statistics.median(r.kernel_ms for r in res)
    r = res[-1]
    c, se = r.row(W3D["target"])[1:]
    info = L.info
    # clearance queries, 1e7 uniform points (inputs + outputs 400 MB, larger than L2)
    rng = np.random.default_rng(0x3D)
    bd = L.bounds
    pts = torch.as_tensor(bd[:3] + rng.random((10_000_000, 3)) * (bd[3:] - bd[:3]), device=device)
    d = torch.empty(len(pts), dtype=torch.float64, device=device)
    k = torch.empty(len(pts), dtype=torch.int64, device=device)
    L.query_device(pts, d, k, stream.cuda_stream)
    e0.record(stream)
    for _ in range(5):
        L.query_device(pts, d, k, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    qms = e0.elapsed_time(e1) / 5
    del pts, d, k
    L.close()
    # end to end: boxes from the host, grid build, walks, rows back, every step
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(steps):
        with frw.Layout3.from_boxes(b, device=device) as Le:
            Le.walk(W3D["target"], W3D["walks"], 500 + i, o, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / steps
    # algorithmic bytes per hop: the cell record, the cell's candidate list
    # (32 B per entry, mean over cells) and one CDF threshold
    bh = 8 + 32 * info.mean_list + 4
    hops = r.hops_total
    peak, peak_kind = measured_peak_hbm()
    ach = hops * bh / (kms * 1e-3) / 1e9
    prof3 = profile_figures(PROFILE3)
    roof3 = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
             "traffic": prof3.get("dram_bytes_per_launch"),
             "note": f"k_walk3; algorithmic {bh:.0f} B/hop x {hops / W3D['walks']:.2f} hops/walk; peak {peak_kind}; "
                     "traffic = DRAM bytes of one 1e6-walk launch under ncu (cold reads of the lists and tables, "
                     "which stay L2-resident: HBM is an upper-bound denominator, issue_frac the bound)"}
    if "warp_instructions_per_walk" in prof3 and sm_mhz:
        sms = torch.cuda.get_device_properties(device).multi_processor_count
        roof3["issue_frac"] = (W3D["walks"] / (kms * 1e-3)) * prof3["warp_instructions_per_walk"] / (
            sms * 4 * sm_mhz * 1e6)
        roof3["warp_instructions_per_walk"] = prof3["warp_instructions_per_walk"]
        roof3["threads_per_instruction"] = prof3.get("threads_per_instruction")
    out = {"workload": W3D["workload"], "config": W3D, "ms_per_step": ms, "walks_per_s": W3D["walks"] / (ms * 1e-3),
           "kernel_ms": kms, "kernel_walks_per_s": W3D["walks"] / (kms * 1e-3),
           "hops_per_s": r.hops_total / (kms * 1e-3), "mean_hops": r.hops_total / W3D["walks"],
           "escaped": int(r.escaped), "c00": c, "c00_rel_se": se / abs(c), "conductors_reached": int(len(r.conductor)),
           "grid": list(info.grid), "grid_build_ms": info.build_ms, "mean_list": info.mean_list,
           "max_list": info.max_list,
           "queries_1e7": {"ms": qms, "queries_per_s": 1e7 / (qms * 1e-3)},
           "roofline": roof3,
           "e2e": {"value": W3D["walks"] / e2e_s, "unit": "walks/s", "h2d_bytes_per_step": W3D["boxes"] * 24,
                   "d2h_bytes_per_step": (5 + 3 * W3D["boxes"]) * 8}}
    if cpu_seconds > 0 and cores > 0:
        ctx = mp.get_context("spawn")
        with ctx.Pool(cores) as pool:
            rs = pool.map(_port3_worker, [(b, W3D["target"], cpu_seconds, i) for i in range(cores)])
        done = sum(x for x, _ in rs)
        out["cpu_port"] = {"value": done / max(t for _, t in rs), "unit": "walks/s", "cores": cores, "kind": "port",
                           "sample": f"the FP64 CPU restatement of the 3-D walk (oracle/frwcpu3d.c, cell grid), "
                                     f"{cpu_seconds:g}s on {cores} processes, {done} walks"}
    return out


# ------------------------------------------------------------ batched config
BATCHED = dict(workload="frw-c4-256-layouts-1e8-walks", layouts=256, min_rects=100, max_rects=100_000,
               total_walks=100_000_000, layout_seed=0x0C4, tune_walks=5_000_000)


def batched_run(frw, device, stream, steps):
    """256 layouts (log-uniform 100..1e5 rects), one target each, walks
    proportional to rects (1e8 in total): one graph-captured persistent launch
    per run, launch parameters from the autotuner."""
    import torch

    B = BATCHED
    rng = np.random.default_rng(B["layout_seed"])
    counts = np.exp(rng.uniform(np.log(B["min_rects"]), np.log(B["max_rects"]), B["layouts"])).astype(int)
    t0 = time.perf_counter()
    layouts = []
    for i, n in enumerate(counts):
        dom = float(np.sqrt(n) * 100.0)  # the configs' density: 1e4 rects on [0,1e4]^2
        layouts.append(frw.Layout.from_rects(frw.generate_layout(B["layout_seed"] + i, int(n), dom), device=device))
    t_layouts = time.perf_counter() - t0
    walks = np.maximum(1, np.round(counts / counts.sum() * B["total_walks"])).astype(np.uint64)
    o = frw.capacitance_opts(1.0)
    batch = frw.Batch(layouts, np.zeros(len(layouts), dtype=np.int64), walks, o)
    t0 = time.perf_counter()
    tuning = batch.tune(B["tune_walks"])
    t_tune = time.perf_counter() - t0
    batch.run(seed=1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        res = batch.run(seed=10 + k)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    total = int(walks.sum())
    out = {"workload": B["workload"], "rects_total": int(counts.sum()), "walks_per_run": total,
           "ms_per_run": ms, "walks_per_s": total / (ms * 1e-3), "tuning": tuning.as_dict(),
           "tune_s": t_tune, "layout_build_s": t_layouts,
           "mean_hops": float(sum(r.hops_total for r in res) / total)}
    batch.close()
    for L in layouts:
        L.close()
    return out


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
    ap.add_argument("--no-headline", action="store_true", help="skip the time-to-0.1%% plain vs CV runs")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-layout batched runs")
    ap.add_argument("--no-3d", action="store_true", help="skip the 3-D walk runs")
    ap.add_argument("--no-sub", action="store_true", help="skip the C2 / C3-capacitance / query sub-lines")
    args = ap.parse_args()
    if args.walks:
        WORKLOAD["walks"] = args.walks
    if args.impl == "reference":
        return run_reference(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # CPU baseline first (spawned pools, before any GPU work), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baselines(args.cpu_seconds)

    import torch

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
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    o = frw.opts(stream_id=shard.plan(W["walks"], rank)["stream"])  # the reference's walk definition
    frw.Layout.from_rects(rects, device=local).close()  # the first build grows the memory pool
    L = frw.Layout.from_rects(rects, device=local)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    # the step's rows stay on the device: hits | stats (int64) and sum_w | sum_w2
    # (float64), cleared per step, summed over ranks by the one exchange
    n = L.n
    rows_i = torch.zeros(n + 4, dtype=torch.int64, device=dev)
    rows_f = torch.zeros(2 * n, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    if dist is not None:  # the exchange: each rank's nonzero rows, all-gathered (NCCL), summed on every rank
        cap = min(n, 1 << 16)
        sbuf = shard.sparse_buffer(cap, dev)
        s_count, s_stats, s_idx, s_hits, s_w, s_w2 = shard.sparse_views(sbuf, cap)
        sum_i, sum_f = torch.zeros_like(rows_i), torch.zeros_like(rows_f)
        overflow = torch.zeros((), dtype=torch.bool, device=dev)

    def step(seed, kev=None):
        rows_i.zero_()
        rows_f.zero_()
        if kev:
            kev[0].record(stream)
        L.walk_device(W["target"], W["walks"], seed, o, rows_i[:n], rows_f[:n], rows_f[n:], rows_i[n:], status,
                      stream.cuda_stream)
        if kev:
            kev[1].record(stream)
        if dist is not None:
            L.rows_compact(rows_i[:n], rows_f[:n], rows_f[n:], s_idx, s_hits, s_w, s_w2, s_count,
                           stream.cuda_stream)
            s_stats.copy_(rows_i[n:])
            g = shard.gather_sparse(sbuf, world)
            sum_i.zero_()
            sum_f.zero_()
            overflow.logical_or_(shard.merge_sparse(g, n, cap, sum_i, sum_f))

    for i in range(args.warmup):
        step(1000 + i)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with Clocks(local) as clk:
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            step(i, kev[i])
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    if int(status.item()) != 0:
        raise RuntimeError(f"walk kernel reported status {int(status.item()):#x}")
    if dist is not None and bool(overflow.item()):
        raise RuntimeError(f"a rank reached more than {cap} conductors in one step: sparse exchange too small")
    kern_ms = [a.elapsed_time(b) for a, b in kev]
    t_ms = sum(a.elapsed_time(b) for a, b in ev)
    if dist is not None:
        t = torch.tensor([t_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    last_i = (rows_i if dist is None else sum_i).cpu().numpy()  # the last step, all ranks
    stats = last_i[n:]
    assert int(stats[3]) == W["walks"] * world, stats
    walks_total = W["walks"] * args.steps * world
    value = walks_total / (t_ms * 1e-3)

    # e2e through the public ABI from pinned host memory, every step:
    # layout upload + tree and cell-list build + walks + rows back
    pinned = torch.from_numpy(rects).pin_memory()
    ptr = pinned.data_ptr()
    import ctypes

    def e2e_step(seed):
        h = ctypes.c_void_p()
        frw._check(frw.lib().frw_layout_create(ctypes.cast(ptr, frw._F), W["rects"], None, local,
                                               ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        Le = frw.Layout(h, W["rects"])
        # room for 65,536 result rows (a step reaches a few hundred conductors; checked below)
        r = Le.walk(W["target"], W["walks"], seed, o, capacity=1 << 16, stream=stream.cuda_stream)
        Le.close()
        assert r.extra["n_entries"] == len(r.conductor), "result rows truncated"
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

    solo = rank == 0 and world == 1
    sub = {}
    if solo and not args.no_sub:
        sub["collision_queries"] = query_rates(frw, L, dev, stream, [("c3_batch_1e7", 10_000_000, 0x0C3, 5)])
    L.close()
    if solo and not args.no_sub:
        sub["c2"] = device_rows_run(frw, C2, frw.capacitance_opts(1.0), local, stream, 10, flush)
        with frw.Layout.from_rects(frw.generate_layout(C2["layout_seed"], C2["rects"], C2["domain"]),
                                   device=local) as L2:
            sub["collision_queries"].update(query_rates(frw, L2, dev, stream,
                                                        [("c2_check_1e5", 100_000, 0x0C2, 20),
                                                         ("c2_batch_1e7", 10_000_000, 0x0C2 + 1, 5)]))
        sub["c3_capacitance"] = device_rows_run(frw, C3CAP, frw.capacitance_opts(1.0), local, stream, 5, flush)
    if solo and not args.no_headline:
        sub["time_to_0.1pct_rel_se"] = time_to_rel_se(frw, local, stream)
    if solo and not args.no_batched:
        sub["batched"] = batched_run(frw, local, stream, 3)
    if solo and not args.no_3d:
        sub["walk3d"] = walk3d_run(frw, local, stream, 3, 0.0 if args.no_cpu_baseline else 2.0,
                                   min(host_cores(), 16), clk.summary().get("sm_mhz"))

    if rank == 0:
        hbar = float(stats[2]) / float(stats[3])
        bq = algorithmic_bytes_per_query(W["rects"])
        kms = statistics.median(kern_ms)
        kernel_walks_s = W["walks"] / (kms * 1e-3)
        achieved = kernel_walks_s * hbar * bq / 1e9
        peak, peak_kind = measured_peak_hbm()
        clocks = clk.summary()
        prof = profile_figures()
        traffic = None
        if "dram_bytes_per_launch" in prof and "walks_per_launch" in prof:
            traffic = prof["dram_bytes_per_launch"] * W["walks"] / prof["walks_per_launch"]
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "algorithmic_bytes_per_walk": hbar * bq,
                "note": f"k_walk; algorithmic {bq} B/query (the tree query's bytes at 10^6 rects) x {hbar:.2f} "
                        f"queries/walk; peak {peak_kind}; a cell-list query reads about 40 B instead (cell "
                        "record and two listed rects, L1/L2-resident), so frac can exceed 1: issue_frac is "
                        "the bound the kernel sits on"}
        if "l2_bytes_per_walk" in prof:
            roof["l2_bytes_per_walk"] = prof["l2_bytes_per_walk"]
        if "warp_instructions_per_walk" in prof and clocks.get("sm_mhz"):
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            issue = kernel_walks_s * prof["warp_instructions_per_walk"] / (sms * 4 * clocks["sm_mhz"] * 1e6)
            roof["issue_frac"] = issue
            roof["warp_instructions_per_walk"] = prof["warp_instructions_per_walk"]
            if "threads_per_instruction" in prof:
                roof["threads_per_instruction"] = prof["threads_per_instruction"]
        out = {
            "metric": METRIC, "value": value, "unit": "walks/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(W),
            "stats": {"mean_hops": hbar, "kernel_ms_median": kms, "kernel_walks_per_s": kernel_walks_s,
                      "queries_per_s": kernel_walks_s * hbar, "escaped_last_step": int(stats[0]),
                      "conductors_reached_last_step": int((last_i[:n] > 0).sum()),
                      "fraction_other_last_step": 1.0 - float(last_i[W["target"]]) / float(stats[3]),
                      "parallelism": f"walks x{world}", "query_semantics": "complete (the reference GPU "
                      "traversal's); the reference CPU tree as shipped misses collisions"},
            "e2e": {"value": W["walks"] / (e2e_ms * 1e-3), "unit": "walks/s",
                    "h2d_bytes_per_step": W["rects"] * 16 + 32,
                    "d2h_bytes_per_step": nrows * 32 + 64},
            "gpu_launches": (2 if world == 1 else 3) * args.steps,
            "roofline": roof,
            "clocks": clocks,
        }
        out.update(sub)
        if cpu:
            out["cpu_baseline"] = cpu
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
