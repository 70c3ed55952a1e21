"""Autotuner for the launch parameters that depend on the workload.

Tuned parameters (process-wide library settings, ``flpr_set_tuning``):

* ``spread_item_points`` -- points per spread work item (one CTA of the
  tile-accumulation kernels): small items spread a dense tile over more
  CTAs, large items cut the per-item overhead;
* ``fused_chunk_mb`` -- column-pass output budget of the fused 2-D
  convolution, i.e. how many bandwidths one column pass / row pass pair
  covers (more bandwidths per chunk: more row-pass CTAs, more traffic);

and, for an :class:`~fastlpr_b200.plan.LprPlan`, the number of concurrent
streams inside its CUDA graph.

Each candidate is timed on the caller's own workload with CUDA events (median
of a few repetitions after a warm-up); the best setting is stored in a JSON
cache keyed by a signature of the workload (shapes, sizes, options), so a
workload is tuned once per machine.  Cache file: ``$FASTLPR_B200_CACHE`` or
``~/.cache/fastlpr_b200/autotune.json``.
"""
from __future__ import annotations

import itertools
import json
import os
from typing import Callable, Dict, List, Optional

import numpy as np
import torch

from . import _lib

PARAMS = {"spread_item_points": 0, "fused_chunk_mb": 1}
ITEM_POINTS = (1024, 2048, 4096, 8192)
CHUNK_MB = (192, 384, 768, 1536)


def set_params(values: Dict[str, int]) -> None:
    lib = _lib.load()
    for name, v in values.items():
        if name in PARAMS:
            _lib.check(lib.flpr_set_tuning(PARAMS[name], int(v)), "flpr_set_tuning")


def get_params() -> Dict[str, int]:
    lib = _lib.load()
    return {name: int(lib.flpr_get_tuning(i)) for name, i in PARAMS.items()}


def _cache_path() -> str:
    p = os.environ.get("FASTLPR_B200_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "fastlpr_b200", "autotune.json")


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, value: dict) -> None:
    path = _cache_path()
    data = _load()
    data[key] = value
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home: tuning still applies to this process


def device_key(device: torch.device) -> str:
    props = torch.cuda.get_device_properties(device)
    return f"{props.name}/sm{props.major}{props.minor}/{props.multi_processor_count}"


def time_ms(fn: Callable[[], None], reps: int = 3, device=None) -> float:
    """Median device time of fn() over `reps` calls after one warm-up."""
    fn()
    torch.cuda.synchronize(device)
    ts = []
    for _ in range(reps):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        ts.append(s.elapsed_time(e))
    return float(np.median(ts))


def tune(key: str, candidates: List[dict], measure: Callable[[dict], float],
         force: bool = False) -> dict:
    """Best candidate by `measure` (milliseconds, lower is better), cached
    under `key`; returns {"best": {...}, "ms": ..., "trials": [...]}."""
    if not force:
        hit = _load().get(key)
        if hit is not None:
            return hit
    trials = []
    for c in candidates:
        trials.append({"params": c, "ms": float(measure(c))})
    best = min(trials, key=lambda t: t["ms"])
    out = {"best": best["params"], "ms": best["ms"], "trials": trials}
    _store(key, out)
    return out


def tune_fit(x, y, h, options: Optional[dict] = None, force: bool = False) -> dict:
    """Tune the spread work-item size and the fused-convolution chunk budget
    for cv_fastlpr on this workload, apply the best and return the record."""
    from . import api
    su = api._lpr_setup(x, y, h, options)
    dev = api._device(su.opts)
    G = api._grid_shape(su.opts, su.n, su.d)
    key = "fit|" + "|".join(str(v) for v in (
        device_key(dev), su.d, tuple(int(g) for g in G), su.order, su.dy, su.y_is_complex,
        su.prec, su.bandwidths.shape[0], int(su.opts.get("num_dof_sample", 10)),
        int(np.round(np.log2(max(su.n, 1)))), str(su.opts.get("kernel_type", "gaussian"))))
    saved = get_params()
    cands = [{"spread_item_points": a, "fused_chunk_mb": b}
             for a, b in itertools.product(ITEM_POINTS, CHUNK_MB)]
    if su.d != 2:
        cands = [c for c in cands if c["fused_chunk_mb"] == saved["fused_chunk_mb"]]
    xd = torch.from_numpy(np.ascontiguousarray(su.x_arr)).to(dev)
    real = not su.y_is_complex and not su.variance

    def run():
        if real:
            api.cv_fastlpr_device(xd, yd, su.bandwidths, su.opts)
        else:
            api.cv_fastlpr(su.x_arr, su.y_arr, su.bandwidths, su.opts)

    yd = torch.from_numpy(np.ascontiguousarray(su.y_arr)).to(dev) if real else None

    def measure(c):
        set_params(c)
        return time_ms(run, device=dev)

    try:
        rec = tune(key, cands, measure, force=force)
    finally:
        set_params(saved)
    set_params(rec["best"])
    return rec
