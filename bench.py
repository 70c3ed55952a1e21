"""Benchmark: bandwidth-selected 2-D local-linear fits per second.

Workload (one "step" = one full GCV sweep = one fit): N = 1e6 points
x ~ U[0,1]^2, y = sin(2 pi x1) cos(2 pi x2) + 0.1 N(0,1), order 1, grid 512^2,
32 isotropic bandwidths log-spaced in [0.005, 0.5] (z-units), 10 Hutchinson
probes, GCV selection.  Synthetic seeded data; every rank fits its own data
set (weak scaling, no collective on the data path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0.  ``value`` is measured with the inputs
resident in HBM (``cv_fastlpr_device``); ``e2e`` goes through the public
``cv_fastlpr`` with pinned host arrays, host->device and device->host copies
inside the timed region.  ``--impl reference`` times the CPU oracle (a
restatement of the reference algorithm) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "2D local-linear fits/s (N=1e6, 32 h) learned vs plain GCV sweep, rel err ≤1e-5"
N_POINTS = 1_000_000
GRID = [512, 512]
N_H = 32
H_RANGE = (0.005, 0.5)
R_PROBES = 10


def workload(seed: int, n: int = N_POINTS):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 2))
    y = np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]) + 0.1 * rng.standard_normal(n)
    hv = np.logspace(np.log10(H_RANGE[0]), np.log10(H_RANGE[1]), N_H)
    h = np.column_stack([hv, hv])
    opts = {"order": 1, "N": list(GRID), "num_dof_sample": R_PROBES}
    return x, y, h, opts


def batched_workload(seed: int = 7, count: int = 512, y_seed: int = 0):
    """The batched uneven workload: `count` independent problems, half 1-D
    (grid 1024) and half 2-D (grid 256^2), N lognormal (median 5e4, sigma 1)
    clipped to [1e3, 1e6], orders drawn from {0, 1, 2}, 25% complex
    responses y = exp(i 2 pi x1) + complex Gaussian noise (sigma 0.1), the
    rest sums of 1-4 random sinusoids plus N(0, 0.1^2) noise, 24 isotropic
    bandwidths in [0.005, 0.5].  The designs x depend on `seed` only; the
    noise of the responses also on `y_seed`."""
    rng = np.random.default_rng(seed)
    hv = np.logspace(np.log10(0.005), np.log10(0.5), 24)
    probs = []
    for k in range(count):
        d = 1 if k % 2 == 0 else 2
        n = int(np.clip(np.round(5e4 * np.exp(rng.standard_normal())), 1e3, 1e6))
        order = int(rng.integers(0, 3))
        cplx = rng.random() < 0.25
        x = rng.random((n, d))
        nsin = int(rng.integers(1, 5))
        freqs = rng.uniform(0.5, 6.0, (nsin, d))
        phases = rng.uniform(0, 2 * np.pi, nsin)
        amps = rng.uniform(0.5, 1.5, nsin)
        ry = np.random.default_rng([seed, k, y_seed])
        if cplx:
            y = np.exp(2j * np.pi * x[:, 0]) + 0.1 * (ry.standard_normal(n)
                                                       + 1j * ry.standard_normal(n))
        else:
            y = sum(a * np.sin(2 * np.pi * (x @ f) + ph) for a, f, ph in zip(amps, freqs, phases))
            y = y + 0.1 * ry.standard_normal(n)
        opts = {"order": order, "N": 1024 if d == 1 else [256, 256]}
        probs.append((x, y, np.column_stack([hv] * d), opts))
    return probs


def b_fit(n=N_POINTS, d=2, G=512, H=N_H, R=R_PROBES, order=1, cy=1, parts=False):
    """Compulsory HBM bytes of one FFT-convolution fit (per-unit figure of the
    roofline): point passes, grid spread/FFT, inverse-pass intermediates and
    the m grids.  parts=True returns the four terms."""
    L = 2 ** int(np.ceil(np.log2(2 * G - 1)))
    nt = 1 + d if order == 1 else (1 if order == 0 else 1 + d + d * (d + 1) // 2)
    ns = nt * (nt + 1) // 2
    C = 2 + R
    P = ns + nt * (1 + R)
    pts = 2 * n * (4 * d + 4 * cy + 8 * R)
    grids = C * L ** d * (4 + 12 + 8)
    inter = sum(H * P * G ** k * L ** (d - k) * 8 * 2 for k in range(1, d))
    mgr = H * (1 + R) * G ** d * 4 * 2
    if parts:
        return {"points": pts, "grids": grids, "intermediates": inter, "m": mgr}
    return pts + grids + inter + mgr


# DRAM traffic of the fused convolution stage of one metric fit
# (dram__bytes_read.sum + dram__bytes_write.sum over its kernels, bytes), from
# an ncu capture of `bench.py --single-fit --points 100000` (the stage works
# on grid-sized arrays only, so the N=1e5 capture holds for N=1e6).
CONV_STAGE_TRAFFIC = 3.396e9


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up (driver queries) must not overlap the
            # timed region: wait for its first sample
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines = []
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [s.strip() for s in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle restatement of the reference path
# ---------------------------------------------------------------------------
def cpu_fit(seed: int, n: int = N_POINTS, workers: int = 0):
    """One full fit of the metric workload (all 32 bandwidths) by the CPU
    oracle on the host cores: (seconds, oracle result, phase seconds)."""
    import oracle
    x, y, h, opts = workload(seed, n)
    workers = workers or (os.cpu_count() or 1)
    t = {}
    t0 = time.perf_counter()
    o = oracle.cv_fastlpr(x, y, h, opts, workers=workers, timings=t)
    return time.perf_counter() - t0, o, t


def cpu_baseline(seed: int, n: int = N_POINTS):
    """Fits/s of the CPU oracle on the metric workload: one full fit (all 32
    bandwidths, the data set the GPU arm fits), timed as a whole."""
    workers = os.cpu_count() or 1
    sec, o, t = cpu_fit(seed, n, workers)
    return {"value": 1.0 / sec, "unit": "fits/s", "cores": workers, "kind": "port",
            "sample": (f"one full fit of the benchmark workload by the CPU oracle (numpy/scipy "
                       f"restatement of the reference path, C gridding): N=1e6, grid 512^2, all "
                       f"32 bandwidths, data seed {seed} (the GPU arm's data), {sec:.1f} s"),
            "seconds_per_fit": sec, "phase_seconds": {k: round(v, 3) for k, v in t.items()},
            "oracle": o}


# ---------------------------------------------------------------------------
# Parity against the CPU oracle: largest relative errors of every output
# (max-normalised for arrays, element-wise for GCV/LCV scores).  Used by the
# cpu_baseline leg of the benchmark and by the configuration parity tests.
# ---------------------------------------------------------------------------
TOL = {"fp32": 1e-5, "fp64": 1e-9}


def _rel(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    den = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0)) if b.size else 0.0


def _erel(a, b) -> float:
    a, b = np.asarray(a, dtype=complex), np.asarray(b, dtype=complex)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def lpr_parity(r, o, tol: float) -> dict:
    """RegressionOutput `r` against the oracle's result `o` of the same fit."""
    e = {"yhat": _rel(r.yhat, o["yhat"]),
         "grid_values": _rel(r.fpp_yhat.values, o["grid_values"]),
         "gcv": _erel(r.gcv_yhat["gcv_m"], o["gcv_m"]),
         "dof": _rel(r.gcv_yhat["dof"], o["dof_all"]),
         "s0": _rel(r.s0, o["s0"])}
    if o.get("d") is not None:
        e["variance_scale"] = abs(r.d - o["d"]) / abs(o["d"])
    same = bool(r.gcv_yhat["id1se"] == o["id1se"])
    worst = max(e.values())
    return {"max_rel_err": worst, "tol": tol, "same_bandwidth": same,
            "ok": bool(worst <= tol and same), **e}


def kde_parity(k, o, tol: float) -> dict:
    e = {"density": _rel(k.metadata["fhat_all"], o["fhat_all"]),
         "lcv": _erel(k.lcv["lcv_m"], o["lcv_m"])}
    same = bool(k.lcv["id1se"] == o["id1se"])
    worst = max(e.values())
    return {"max_rel_err": worst, "tol": tol, "same_bandwidth": same,
            "ok": bool(worst <= tol and same), **e}


def hetero_bandwidth_sample(H: int, sel: int, count: int = 6) -> np.ndarray:
    """Bandwidth indices of the 2-D local-quadratic parity case: the
    smallest, the largest, the full sweep's choice and its neighbours, filled
    up evenly to `count`."""
    idx = {0, H - 1, sel, max(sel - 1, 0), min(sel + 1, H - 1)}
    for v in np.linspace(0, H - 1, count).round().astype(int):
        if len(idx) >= count:
            break
        idx.add(int(v))
    return np.array(sorted(idx))


def batched_sample(count: int = 16):
    """The first `count` problems of the batched workload (1-D and 2-D,
    orders 0-2, complex responses, N from 9e3 to 8.3e5 for 16)."""
    return batched_workload(count=512)[:count]


def parity_hetero2d(dev, workers: int, full_sel: int = None):
    """2-D local-quadratic heteroscedastic configuration at full size
    (N = 2e6, grid 512^2) on a sample of its 32 bandwidths: the mean fit,
    then the variance fit of the squared residuals, GPU (default precision:
    FP32 value channels, FP64 moment planes and solves) against the oracle
    on identical inputs, each at the tolerance of the precision it ran in."""
    import fastlpr_b200
    import oracle
    x, y, h, o = config_workloads()["lpr2d_o2_hetero"]
    opts = dict(o, device=str(dev))
    if full_sel is None:
        full_sel = int(fastlpr_b200.cv_fastlpr(x, y, h, opts).gcv_yhat["id1se"])
    hs = h[hetero_bandwidth_sample(len(h), full_sel)]
    r = fastlpr_b200.cv_fastlpr(x, y, hs, opts)
    om = oracle.cv_fastlpr(x, y, hs, o, workers=workers)
    yv = (y - r.yhat) ** 2
    v = fastlpr_b200.cv_fastlpr(x, yv, hs, dict(opts, y_type_out="variance"))
    ov = oracle.cv_fastlpr(x, yv, hs, dict(o, y_type_out="variance"), workers=workers)
    return {"mean": lpr_parity(r, om, TOL[r.metadata["precision"]]),
            "variance": lpr_parity(v, ov, TOL[v.metadata["precision"]]),
            "bandwidths": [int(i) for i in hetero_bandwidth_sample(len(h), full_sel)],
            "points": int(x.shape[0]), "precision": r.metadata["precision"],
            "moment_planes": r.metadata.get("moment_planes"),
            "fp64_bandwidths": int(r.metadata.get("fp64_bandwidths", 0))}


def parity_lpr1d(dev, workers: int):
    """1-D local-linear configuration at full size (N = 1e5, grid 1024,
    20 bandwidths), default precision (FP32 grids)."""
    import fastlpr_b200
    import oracle
    x, y, h, o = config_workloads()["lpr1d"]
    r = fastlpr_b200.cv_fastlpr(x, y, h, dict(o, device=str(dev)))
    return dict(lpr_parity(r, oracle.cv_fastlpr(x, y, h, o, workers=workers), TOL["fp32"]),
                precision=r.metadata["precision"])


def parity_kde3d(dev, workers: int, n: int = 1_000_000):
    """3-D KDE configuration (mixture of 8 anisotropic Gaussians plus 10%
    uniform background, grid 128^3, 16 bandwidths) at N = 1e6 points."""
    import fastlpr_b200
    import oracle
    x, h, o = kde3d_workload(n)
    k = fastlpr_b200.cv_fastkde(x, h, dict(o, device=str(dev)))
    return dict(kde_parity(k, oracle.cv_fastkde(x, h, o, workers=workers), TOL["fp32"]),
                points=n, precision=k.metadata["precision"])


def parity_batched(results, probs, workers: int) -> dict:
    """Batched-workload results (RegressionOutputs of `probs`, in order)
    against the oracle, problem by problem; worst case per precision."""
    import oracle
    out = {}
    for k, (r, (x, y, h, o)) in enumerate(zip(results, probs)):
        prec = r.metadata["precision"]
        p = lpr_parity(r, oracle.cv_fastlpr(x, y, h, o, workers=workers), TOL[prec])
        q = out.setdefault(prec, {"problems": 0, "max_rel_err": 0.0, "tol": TOL[prec],
                                  "all_same_bandwidth": True, "ok": True})
        q["problems"] += 1
        if p["max_rel_err"] >= q["max_rel_err"]:
            fields = {f: v for f, v in p.items()
                      if isinstance(v, float) and f not in ("tol", "max_rel_err")}
            q["worst"] = {"problem": k, "field": max(fields, key=fields.get),
                          "fp64_bandwidths": int(r.metadata.get("fp64_bandwidths", 0))}
        q["max_rel_err"] = max(q["max_rel_err"], p["max_rel_err"])
        q["all_same_bandwidth"] = q["all_same_bandwidth"] and p["same_bandwidth"]
        q["ok"] = q["ok"] and p["ok"]
    return out


# ---------------------------------------------------------------------------
def _dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def replica_seed(rank: int) -> int:
    """Seed of the data set a rank fits: every replica has its own data."""
    return 1000 + rank


def max_over_ranks(ms: float, world: int, device) -> float:
    """The slowest rank's elapsed time (the job's time for weak scaling)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def bench_config(world: int) -> dict:
    """The `config` of the benchmark line (both arms print the same one)."""
    return {"workload": "2-D local-linear GCV sweep (plain full sweep), N=1e6, grid 512^2, "
                        "32 isotropic h in [0.005,0.5], 10 Hutchinson probes",
            "global_batch": world, "parallelism": f"replicas x{world}",
            "l2": "working set (spectra, S/T planes) far larger than the 126 MB L2"}


def run_reference(args):
    """The reference path on the host cores: every step is one full fit of
    the benchmark workload (all 32 bandwidths, the data set rank 0 of the GPU
    arm fits) by the CPU oracle, with all host cores; W warm-up fits first.
    Rank 0 alone runs and prints under torchrun."""
    world, rank, _ = _dist_env()
    if rank != 0:
        return 0
    seed = replica_seed(0)
    workers = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_fit(seed, workers=workers)
    secs = [cpu_fit(seed, workers=workers)[0] for _ in range(max(1, args.steps))]
    total = sum(secs)
    v = len(secs) / total
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "fits/s",
        "n_gpus": args.gpus,
        "steps": len(secs),
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / len(secs),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded numpy), x~U[0,1]^2, y=sin(2pi x1)cos(2pi x2)+0.1N(0,1)",
        "config": bench_config(args.gpus),
        "cpu_baseline": {"value": v, "unit": "fits/s", "cores": workers, "kind": "port",
                         "sample": (f"{len(secs)} full fits of the benchmark workload (all 32 "
                                    f"bandwidths, data seed {seed}) by the CPU oracle on "
                                    f"{workers} host threads, after {args.warmup} warm-up fits; "
                                    f"median {statistics.median(secs):.2f} s per fit")},
        "e2e": {"value": v, "unit": "fits/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "seconds_per_fit": [round(t, 3) for t in secs],
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batched(args, dev, world: int = 1, rank: int = 0, barrier=lambda: None,
                keep: dict = None):
    """The batched uneven workload through LprPlan: every problem's
    y-dependent work captured in one CUDA graph over concurrent streams and
    replayed; each step replaces all responses (fresh noise, pinned staging,
    host-to-device copies inside the timed region) and returns every
    RegressionOutput.  Compared with one cv_fastlpr call per problem.  With
    several ranks the problems are split between them by estimated cost and
    the batch time is the slowest rank's (no other collective)."""
    import torch

    import fastlpr_b200
    from fastlpr_b200.plan import estimated_cost, partition_by_cost
    count = args.batched
    allp = batched_workload(count=count)
    ally = batched_workload(count=count, y_seed=1)
    mine = partition_by_cost([estimated_cost(*p) for p in allp], world)[rank]
    probs = [allp[i] for i in mine]
    ys = [[p[1] for p in probs], [ally[i][1] for i in mine]]
    t0 = time.perf_counter()
    plan = fastlpr_b200.LprPlan(probs, device=dev)
    build_s = time.perf_counter() - t0
    res = None
    for k in range(3):
        res = plan.run(ys[k % 2])
    torch.cuda.synchronize(dev)
    steps = max(2, min(args.steps, 5))
    barrier()
    t0 = time.perf_counter()
    for k in range(steps):
        res = plan.run(ys[k % 2])
    ms = max_over_ranks(1000.0 * (time.perf_counter() - t0) / steps, world, dev)
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record()
    plan.replay()
    e.record()
    e.synchronize()
    replay_ms = s.elapsed_time(e)
    barrier()
    t0 = time.perf_counter()
    for (x, y, h, o) in probs:
        fastlpr_b200.cv_fastlpr(x, y, h, o)
    torch.cuda.synchronize(dev)
    seq_ms = max_over_ranks(1000.0 * (time.perf_counter() - t0), world, dev)
    npts = int(sum(p[0].shape[0] for p in allp))
    if keep is not None:
        # one more run on the first responses: its results, in problem order,
        # for the parity check of the cpu_baseline leg
        keep["results"] = plan.run(ys[0])
        keep["problems"] = probs
    return {
        "workload": (f"{count} independent problems: half 1-D (grid 1024), half 2-D (grid 256^2), "
                     "N lognormal median 5e4 clipped [1e3,1e6], orders 0-2, 25% complex, 24 h; "
                     "full GCV sweep each"),
        "points": npts,
        "value": count * 1000.0 / ms, "unit": "fits/s", "ms_per_batch": ms,
        "graph_replay_ms": replay_ms,
        "sequential_fits_per_s": count * 1000.0 / seq_ms,
        "speedup_vs_sequential": seq_ms / ms,
        "streams": len(plan.streams), "plan_build_s": build_s,
        "ranks": world, "problems_per_rank": len(probs),
        "timing": "wall clock per step (host staging, replay, reductions, outputs) with the previous step's results held, after 3 warm-up steps",
    }


def run_learned_batched(args, dev, plain_fits_per_s: float):
    """The learned search over a batch of benchmark-shaped data sets (N = 1e6,
    grid 512^2, the 32 bandwidths, each its own seed) through one LprPlan:
    binned sums, features, the network (one batch) and every window chosen
    and evaluated inside one CUDA graph; each step stages new responses for
    every data set (host-to-device copies inside the timed region), replays
    and returns every result.  The same data sets through a full-sweep
    LprPlan give the swept GCV optimum each choice is judged against."""
    import torch

    import fastlpr_b200
    count = args.learned_batched
    probs, ys2 = [], []
    for k in range(count):
        x, y, h, o = workload(2000 + k)
        rng = np.random.default_rng(3000 + k)
        probs.append((x, y, h, dict(o, precision="fp32", bandwidth_search="learned")))
        ys2.append(np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1])
                   + 0.1 * rng.standard_normal(x.shape[0]))
    ys = [[p[1] for p in probs], ys2]
    t0 = time.perf_counter()
    plan = fastlpr_b200.LprPlan(probs, device=dev)
    build_s = time.perf_counter() - t0
    try:
        # warm-up as the timed steps run: the caller holds the previous
        # step's results (their pinned pages) while the next step runs
        res = None
        for k in range(3):
            res = plan.run(ys[k % 2])
        torch.cuda.synchronize(dev)
        steps = max(2, min(args.steps, 5))
        t0 = time.perf_counter()
        for k in range(steps):
            res = plan.run(ys[k % 2])
        ms = 1000.0 * (time.perf_counter() - t0) / steps
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        plan.replay()
        e.record()
        e.synchronize()
        replay_ms = s.elapsed_time(e)
        last = plan.run(ys[0])
    finally:
        plan.close()
    # the full sweep of the same data sets judges every choice
    fprobs = [(x, y, h, dict(o, bandwidth_search="full")) for (x, y, h, o) in probs]
    fplan = fastlpr_b200.LprPlan(fprobs, device=dev)
    try:
        fplan.run(ys[0])
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        full = fplan.run(ys[0])
        full_ms = 1000.0 * (time.perf_counter() - t0)
    finally:
        fplan.close()
    ratios, accepted, evaluated, same = [], 0, [], 0
    for lr, fr in zip(last, full):
        bs = lr.metadata["bandwidth_search"]
        accepted += int(bool(bs.get("accepted")))
        evaluated.append(int(bs.get("evaluated", len(fr.gcv_yhat["gcv_m"]))))
        ratios.append(float(np.min(lr.gcv_yhat["gcv_m"]) / np.min(fr.gcv_yhat["gcv_m"])))
        same += int(np.allclose(lr.h, fr.h))
    value = count * 1000.0 / ms
    return {
        "workload": (f"{count} data sets of the benchmark shape (N=1e6, grid 512^2, 32 isotropic h "
                     f"in [0.005,0.5], 10 probes, seeds 2000..{1999 + count}), learned search in "
                     "one LprPlan graph; new responses every step"),
        "value": value, "unit": "fits/s", "ms_per_batch": ms, "graph_replay_ms": replay_ms,
        "speedup_vs_plain": value / plain_fits_per_s,
        "full_sweep_batched_fits_per_s": count * 1000.0 / full_ms,
        "speedup_vs_full_sweep_batched": full_ms / ms,
        "accepted": accepted, "bandwidths_evaluated_mean": float(np.mean(evaluated)),
        "gcv_ratio_vs_full_sweep_max": float(np.max(ratios)),
        "all_within_1pct_gcv": bool(np.max(ratios) <= 1.01),
        "same_bandwidth_as_full_sweep": same, "plan_build_s": build_s,
        "timing": "wall clock per step (staging, replay, outputs) with the previous step's results held, after 3 warm-up steps",
    }


def kde3d_workload(n: int, seed: int = 5):
    """The 3-D KDE case: a mixture of 8 anisotropic Gaussians (means
    U[0.2,0.8]^3, per-axis std U[0.02,0.1], equal weights) plus 10% uniform
    background on [0,1]^3; grid 128^3, 16 isotropic h in [0.01, 0.3]."""
    rng = np.random.default_rng(seed)
    nb = n // 10
    means = rng.uniform(0.2, 0.8, (8, 3))
    sds = rng.uniform(0.02, 0.1, (8, 3))
    comp = rng.integers(0, 8, n - nb)
    x = np.vstack([means[comp] + sds[comp] * rng.standard_normal((n - nb, 3)), rng.random((nb, 3))])
    hv = np.logspace(np.log10(0.01), np.log10(0.3), 16)
    return x, np.column_stack([hv] * 3), {"N": [128, 128, 128]}


def config_workloads():
    """The other configurations, at full size (seeded synthetic data):
    'lpr1d'  1-D local linear, N = 1e5, x ~ U[0,1], y = sin 2 pi x + 0.1 N(0,1),
             grid 1024, 20 h in [0.01, 1];
    'lpr2d_o2_hetero'  2-D local quadratic, N = 2e6, x ~ U[0,1]^2,
             y = sin(2 pi x1) cos(2 pi x2) + (0.05 + 0.1 x1) N(0,1), grid 512^2,
             32 isotropic h in [0.005, 0.5], then the variance fit of the
             squared residuals (order 2, y_type_out 'variance') on the same h;
    'kde3d'  3-D KDE, N = 1e7 (kde3d_workload), grid 128^3, 16 h."""
    rng = np.random.default_rng(11)
    x1 = rng.random(100_000)
    y1 = np.sin(2 * np.pi * x1) + 0.1 * rng.standard_normal(x1.size)
    h1 = np.logspace(-2, 0, 20)[:, None]
    rng = np.random.default_rng(12)
    x2 = rng.random((2_000_000, 2))
    y2 = (np.sin(2 * np.pi * x2[:, 0]) * np.cos(2 * np.pi * x2[:, 1])
          + (0.05 + 0.1 * x2[:, 0]) * rng.standard_normal(x2.shape[0]))
    hv = np.logspace(np.log10(0.005), np.log10(0.5), 32)
    h2 = np.column_stack([hv, hv])
    x3, h3, o3 = kde3d_workload(10_000_000)
    return {"lpr1d": (x1, y1, h1, {"order": 1, "N": [1024]}),
            "lpr2d_o2_hetero": (x2, y2, h2, {"order": 2, "N": [512, 512]}),
            "kde3d": (x3, None, h3, o3)}


def run_configs(args, dev, steps: int = 5, keep: dict = None):
    """Each other configuration through the public API with host arrays
    (cv_fastlpr / cv_fastkde; uploads and downloads included), after two
    warm-up calls: seconds per fit, the median of `steps` calls timed by wall
    clock around synchronised calls."""
    import torch

    import fastlpr_b200
    out = {}
    for name, (x, y, h, o) in config_workloads().items():
        opts = dict(o, device=str(dev))
        try:
            if name == "kde3d":
                def step():
                    return fastlpr_b200.cv_fastkde(x, h, opts)
            elif name == "lpr2d_o2_hetero":
                def step():
                    r = fastlpr_b200.cv_fastlpr(x, y, h, opts)
                    v = fastlpr_b200.cv_fastlpr(x, (y - r.yhat) ** 2, h,
                                                dict(opts, y_type_out="variance"))
                    return r, v
            else:
                def step():
                    return fastlpr_b200.cv_fastlpr(x, y, h, opts)
            step()
            last = step()
            torch.cuda.synchronize(dev)
            times = []
            for _ in range(steps):
                t0 = time.perf_counter()
                step()
                torch.cuda.synchronize(dev)
                times.append(time.perf_counter() - t0)
            if keep is not None:
                keep[name] = last
            sec = float(np.median(times))
            out[name] = {"seconds_per_fit": sec, "fits_per_s": 1.0 / sec, "steps": steps,
                         "points": int(x.shape[0]), "bandwidths": int(len(h))}
        except Exception as e:  # an out-of-memory or unsupported case is reported, not fatal
            out[name] = {"error": f"{type(e).__name__}: {e}"[:200]}
    return out


def run_profile_case(args, dev):
    """One small fit of a kind the benchmark leg does not run, for kernel
    profiles: 'kde3d' (3-D KDE, grid 128^3), 'learned' (learned search on
    the benchmark data), 'cubic2d' (2-D, n = 3000: cubic GCV/DoF), 'order2'
    (2-D local quadratic, FP64 separable convolution), 'hetero2d' (the full
    2-D local-quadratic mean + variance pair of config_workloads),
    'batched64' (the first 64 problems of the batched workload through
    cv_fastlpr_many: the plan's streams and kernels, launched eagerly)."""
    import torch

    import fastlpr_b200
    case = args.profile_case
    t0 = time.perf_counter()
    if case == "kde3d":
        x, h, o = kde3d_workload(args.points)
        r = fastlpr_b200.cv_fastkde(x, h, dict(o, device=str(dev)))
    elif case == "batched64":
        rs = fastlpr_b200.cv_fastlpr_many(batched_workload(count=512)[:64], device=dev)
        r = rs[0]
    elif case == "hetero2d":
        x, y, h, o = config_workloads()["lpr2d_o2_hetero"]
        opts = dict(o, device=str(dev))
        r = fastlpr_b200.cv_fastlpr(x, y, h, opts)
        fastlpr_b200.cv_fastlpr(x, (y - r.yhat) ** 2, h, dict(opts, y_type_out="variance"))
    else:
        n = {"learned": args.points, "cubic2d": 3000, "order2": 50000}[case]
        x, y, h, o = workload(0, n)
        opts = dict(o, device=str(dev))
        if case == "learned":
            opts.update(precision="fp32", bandwidth_search="learned")
        elif case == "cubic2d":
            opts.update(N=[64, 64])
        else:
            opts.update(order=2, N=[256, 256])
        r = fastlpr_b200.cv_fastlpr(x, y, h, opts)
    torch.cuda.synchronize(dev)
    return {"profile_case": case, "seconds": time.perf_counter() - t0,
            "h": [float(v) for v in np.atleast_1d(r.h)]}


def mlp_timing(dev, reps: int = 200) -> dict:
    """Forward pass of the trained proposal network on batches of 1 and
    1024 rows: the one-launch tensor-core kernel (flpr_mlp_infer:
    tcgen05.mma, accumulators in tensor memory) beside the layer-by-layer
    kernels (flpr_mlp_fwd: mma.sync), each the mean of `reps` launches
    timed with CUDA events on the launching stream after warm-up."""
    import torch
    from fastlpr_b200 import _lib
    from fastlpr_b200 import learned as _learned
    lib = _lib.load()
    model = _learned.default_model(dev)
    dims = [int(v) for v in model.dims]
    flops_row = 2.0 * sum(dims[i] * dims[i + 1] for i in range(len(dims) - 1))
    stream = torch.cuda.current_stream(dev)
    out = {"dims": dims, "flops_per_row": flops_row}
    fused_ok = bool(lib.flpr_mlp_infer_supported(model.nl, model._dims_c))
    for rows in (1, 1024):
        x16 = torch.randn((rows, dims[0]), device=dev).to(torch.bfloat16)
        y = torch.empty(rows, dtype=torch.float32, device=dev)
        y2 = torch.empty((rows, 1), dtype=torch.float32, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        ws = torch.empty(lib.flpr_mlp_ws(model.nl, model._dims_c, rows), dtype=torch.uint8,
                         device=dev)

        def tc():
            _lib.check(lib.flpr_mlp_infer(model.nl, model._dims_c, model.p16.data_ptr(),
                                          model.p32.data_ptr(), rows, x16.data_ptr(),
                                          y.data_ptr(), status.data_ptr(), stream.cuda_stream),
                       "flpr_mlp_infer")

        def layers():
            _lib.check(lib.flpr_mlp_fwd(model.nl, model._dims_c, model.p16.data_ptr(),
                                        model.p32.data_ptr(), rows, x16.data_ptr(),
                                        y2.data_ptr(), ws.data_ptr(), ws.numel(),
                                        stream.cuda_stream), "flpr_mlp_fwd")

        rec = {}
        for name, fn in (("tcgen05_one_launch", tc), ("mma_sync_layers", layers)):
            if name == "tcgen05_one_launch" and not fused_ok:
                continue
            for _ in range(10):
                fn()
            torch.cuda.synchronize(dev)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record(stream)
            for _ in range(reps):
                fn()
            e.record(stream)
            e.synchronize()
            us = 1000.0 * s.elapsed_time(e) / reps
            rec[name] = {"us": us, "tflops": flops_row * rows / (us * 1e-6) / 1e12}
        if fused_ok:
            torch.cuda.synchronize(dev)
            rec["status_ok"] = int(status.item()) == 0
        out[f"rows_{rows}"] = rec
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    import fastlpr_b200
    from fastlpr_b200 import _lib

    world, rank, local = _dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    x, y, h, opts = workload(replica_seed(rank), args.points)
    if args.grid:
        opts["N"] = [args.grid, args.grid]
    if args.bandwidths:
        h = h[np.linspace(0, N_H - 1, args.bandwidths).round().astype(int)]
    opts = dict(opts, precision="fp32", device=str(dev))
    # resident inputs
    xd = torch.from_numpy(x).to(dev)
    yd = torch.from_numpy(y).to(dev)
    # pinned host inputs for the end-to-end measurement
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.from_numpy(y).pin_memory()
    xh, yh = xp.numpy(), yp.numpy()

    lib = _lib.load()
    if args.profile_case:
        print(json.dumps(run_profile_case(args, dev)), flush=True)
        return 0
    if args.only_configs:
        print(json.dumps({"configs": run_configs(args, dev)}), flush=True)
        return 0
    if args.only_batched:
        # the batched leg alone (profiling): no metric fits before it
        print(json.dumps(run_batched(args, dev, world, rank, barrier)), flush=True)
        return 0
    if args.single_fit:
        # one plain fit and nothing else: the command profiles are captured with
        l0 = lib.flpr_launch_count()
        t0 = time.perf_counter()
        r = fastlpr_b200.cv_fastlpr_device(xd, yd, h, opts)
        torch.cuda.synchronize()
        print(json.dumps({"single_fit_ms": 1000.0 * (time.perf_counter() - t0),
                          "launches": int(lib.flpr_launch_count() - l0),
                          "h": [float(v) for v in np.atleast_1d(r.h)]}), flush=True)
        return 0
    warm = max(args.warmup, 3)
    counts = {}

    def timed(fn, steps):
        # W untimed steps of this same path right before its timed steps
        # (each path has its own first-call costs: allocator and
        # pinned-memory caches, plans)
        for _ in range(warm):
            fn()
        barrier()
        torch.cuda.synchronize()
        counts["l0"] = lib.flpr_launch_count()
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(steps):
            fn()
        e.record()
        torch.cuda.synchronize()
        counts["launches"] = (lib.flpr_launch_count() - counts["l0"]) // max(1, steps)
        barrier()
        return max_over_ranks(s.elapsed_time(e), world, dev)

    clocks = ClockSampler(local)
    clocks.start()
    res = {}

    def step_dev():
        res["r"] = fastlpr_b200.cv_fastlpr_device(xd, yd, h, opts)

    ms_dev = timed(step_dev, args.steps)
    launches = counts["launches"]

    def step_e2e():
        res["e"] = fastlpr_b200.cv_fastlpr(xh, yh, h, opts)

    ms_e2e = timed(step_e2e, args.steps)
    clk = clocks.stop()

    # per-phase device times of one fit (CUDA events on the launching stream)
    phases = {}
    for _ in range(2):
        fastlpr_b200.cv_fastlpr_device(xd, yd, h, dict(opts, _timings=phases))
    phases = {k: v / 2 for k, v in phases.items()}

    # learned bandwidth search on the same data: proposal + five-bandwidth refine
    learned = None
    try:
        from fastlpr_b200 import learned as _learned
        have_net = os.path.exists(_learned.WEIGHTS_PATH)
    except ImportError:
        have_net = False
    if have_net and not args.bandwidths:
        lopts = dict(opts, bandwidth_search="learned")

        def step_learned():
            res["l"] = fastlpr_b200.cv_fastlpr_device(xd, yd, h, lopts)

        ms_l = timed(step_learned, args.steps)
        full_r, lr_r = res["r"], res["l"]
        bs = lr_r.metadata["bandwidth_search"]
        sel_gcv = float(np.min(lr_r.gcv_yhat["gcv_m"]))
        learned = {
            "value": world * 1000.0 / (ms_l / args.steps), "unit": "fits/s",
            "ms_per_step": ms_l / args.steps,
            "speedup_vs_plain": ms_dev / ms_l,
            "accepted": bool(bs.get("accepted", False)),
            "bandwidths_evaluated": int(bs.get("evaluated", len(h))),
            "gcv_ratio_vs_full_sweep": sel_gcv / float(np.min(full_r.gcv_yhat["gcv_m"])),
            "same_bandwidth_as_full_sweep": bool(np.allclose(lr_r.h, full_r.h)),
            "yhat_max_rel_diff_vs_full_sweep": float(
                np.max(np.abs(lr_r.yhat - full_r.yhat)) / np.max(np.abs(full_r.yhat))),
        }
        learned["network_inference"] = mlp_timing(dev)
    elif not have_net:
        learned = {"unavailable": "no trained bandwidth network (fastlpr_b200/data/bandwidth_mlp.npz)"}

    learned_batched = None
    if args.learned_batched and not args.bandwidths and args.points == N_POINTS and have_net:
        learned_batched = run_learned_batched(args, dev, world * 1000.0 / (ms_dev / args.steps))
    batched = None
    kept_batched, kept_configs = {}, {}
    if args.batched and not args.bandwidths and args.points == N_POINTS:
        batched = run_batched(args, dev, world, rank, barrier, keep=kept_batched)
    # the other configurations, one GPU only (informational, end to end)
    configs = None
    if world == 1 and not args.no_configs and not args.bandwidths and args.points == N_POINTS:
        configs = run_configs(args, dev, keep=kept_configs)

    per_step_ms = ms_dev / args.steps
    value = world * 1000.0 / per_step_ms
    e2e_value = world * 1000.0 / (ms_e2e / args.steps)
    # x, y and the per-bandwidth sums of h for the device-side 1-SE choice
    h2d = x.nbytes + y.nbytes + len(h) * 8
    # fitted values and residuals (float64, n each), selected grid and s0
    # plane (float64, M each), GCV / DoF arrays (4 H float64) and the chosen
    # index (int32)
    M_grid = int(np.prod(opts["N"]))
    d2h = 2 * y.nbytes + 2 * M_grid * 8 + 4 * len(h) * 8 + 4
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    # dominant stage: the fused convolution + solve (column/row-pass FFT
    # kernels), timed with CUDA events on its stream; algorithmic bytes = the
    # inverse-pass intermediates and m terms of B_fit
    bf = b_fit()
    parts = b_fit(parts=True)
    conv_bytes = parts["intermediates"] + parts["m"]
    conv_ms = phases.get("conv_solve")
    achieved_fit = bf / (per_step_ms / 1000.0) / 1e9
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "fits/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": warm,
        "ms_per_step": per_step_ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded numpy), x~U[0,1]^2, y=sin(2pi x1)cos(2pi x2)+0.1N(0,1)",
        "config": bench_config(world),
        "precision": "FP32 grids/FFT/products, FP64 solve and reductions",
        "e2e": {"value": e2e_value, "unit": "fits/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": ({"bound": "hbm", "achieved": conv_bytes / (conv_ms / 1000.0) / 1e9,
                      "peak": hbm, "unit": "GB/s",
                      "frac": conv_bytes / (conv_ms / 1000.0) / 1e9 / hbm,
                      "traffic": CONV_STAGE_TRAFFIC,
                      # what the stage's measured DRAM traffic uses of the peak
                      "traffic_frac": CONV_STAGE_TRAFFIC / (conv_ms / 1000.0) / 1e9 / hbm,
                      "scope": (f"fused convolution + solve stage (colpass/rowpass kernels) of one "
                                f"fit: algorithmic {conv_bytes / 1e9:.2f} GB (B_fit intermediates + "
                                f"m) over {conv_ms:.3f} ms; peak "
                                + ("measured" if "hbm_gbs" in peaks else "fallback"))}
                     if conv_ms else None),
        "roofline_whole_fit": {"achieved": achieved_fit, "peak": hbm, "unit": "GB/s",
                               "frac": achieved_fit / hbm,
                               "algorithmic_bytes": bf},
        "learned": learned,
        "learned_batched": learned_batched,
        "batched": batched,
        "configs": configs,
        "phase_ms": {k: round(v, 3) for k, v in phases.items()},
        "clocks": clk,
    }
    if args.points != N_POINTS or args.grid or args.bandwidths:
        line["config"]["workload"] = (f"profiling case: N={args.points}, grid {opts['N']}, "
                                      f"{len(h)} bandwidths (not the benchmark workload)")
    if (rank == 0 and world == 1 and not args.no_cpu_baseline and not args.grid
            and not args.bandwidths):
        # the CPU oracle on the same data: its timing is the CPU baseline and
        # its outputs are the parity check of the fit timed above; the other
        # configurations are checked against it the same way
        workers = os.cpu_count() or 1
        cb = cpu_baseline(replica_seed(rank), args.points)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        parity = {"metric": dict(lpr_parity(res["r"], cb["oracle"], TOL["fp32"]),
                                 precision="fp32", bandwidths=len(h), points=args.points)}
        if res.get("l") is not None:
            # the learned search's fit against the oracle's full sweep
            parity["metric_learned"] = {
                "yhat": _rel(res["l"].yhat, cb["oracle"]["yhat"]), "tol": TOL["fp32"],
                "same_bandwidth": bool(np.allclose(res["l"].h, cb["oracle"]["h_sel"]))}
        if configs is not None and not args.no_parity:
            parity["lpr1d"] = parity_lpr1d(dev, workers)
            hs = kept_configs.get("lpr2d_o2_hetero")
            parity["lpr2d_o2_hetero"] = parity_hetero2d(
                dev, workers, int(hs[0].gcv_yhat["id1se"]) if hs is not None else None)
            parity["kde3d"] = parity_kde3d(dev, workers)
        if kept_batched.get("results") is not None and not args.no_parity:
            ns = min(16, len(kept_batched["results"]))
            parity["batched_sample"] = parity_batched(kept_batched["results"][:ns],
                                                      kept_batched["problems"][:ns], workers)
        line["parity"] = parity
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def build_parser() -> argparse.ArgumentParser:
    """The command-line options of this benchmark."""
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU oracle (CPU baseline and every parity check)")
    ap.add_argument("--no-parity", action="store_true",
                    help="check only the benchmark fit against the oracle (not the other "
                         "configurations)")
    ap.add_argument("--learned-batched", type=int, default=32,
                    help="data sets of the learned-search batch leg (0: skip)")
    ap.add_argument("--batched", type=int, default=512,
                    help="problems of the batched workload leg (0: skip)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the timing of the other configurations")
    ap.add_argument("--only-configs", action="store_true",
                    help="time only the other configurations (1-D, 2-D order 2 + variance, "
                         "3-D KDE) through the public API")
    ap.add_argument("--only-batched", action="store_true",
                    help="run only the batched workload leg (profiling)")
    ap.add_argument("--profile-case", default="",
                    choices=["", "kde3d", "learned", "cubic2d", "order2", "hetero2d",
                             "batched64"],
                    help="run one small fit of another kind (profiling)")
    ap.add_argument("--single-fit", action="store_true",
                    help="run one plain fit of the workload and exit (for profilers)")
    ap.add_argument("--points", type=int, default=N_POINTS,
                    help="points per fit (profiling of smaller cases only)")
    ap.add_argument("--grid", type=int, default=0, help="grid per axis (default 512)")
    ap.add_argument("--bandwidths", type=int, default=0, help="subset of the 32 bandwidths")
    return ap


def main():
    ap = build_parser()
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
