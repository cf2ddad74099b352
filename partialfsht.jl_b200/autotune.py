"""Tile-shape autotuner for plans.

The device tile shapes of a plan -- rings per lane of the ring passes, NUFFT bin height, degree
segment length of the adjoint ring pass -- change its apply time but not its results. For a
plan's geometry this module times candidate shapes on the device (forward + adjoint, CUDA
events) by coordinate descent and keeps the fastest. Results are cached in a JSON file keyed by
a shape class (lmax and point count in half-octave buckets, tolerance, transforms, precision),
so later plans of the same class are built with the tuned shapes without timing.

    from pfsht_b200 import autotune
    plan = autotune.tuned_plan(theta, phi, lmax=1024, tol=1e-8)
"""
from __future__ import annotations

import json
import math
import os
import threading

CANDIDATES = (
    ("rings_per_lane", (0, 2, 4)),
    ("bin_rows", (0, 16, 32)),
    ("segment_degrees", (0, 512, -1)),
)

_lock = threading.Lock()


def default_cache_path() -> str:
    return os.environ.get("PFSHT_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "pfsht_b200", "tiles.json"))


def shape_class(lmax, npts, tol, ntrans, precision) -> str:
    """Plans whose apply times scale alike share tuned shapes."""
    lb = round(2 * math.log2(max(lmax, 1))) / 2
    nb = round(2 * math.log2(max(npts, 1))) / 2
    bb = 1 if ntrans == 1 else (2 if ntrans < 4 else 4)
    return f"L{lb:g}:M{nb:g}:tol{tol:g}:B{bb}:{precision}"


def _load(path):
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + f".{os.getpid()}.tmp"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_plan(pf, plan, reps=5, warmup=2) -> float:
    """Device time of one forward + adjoint apply of `plan`, in ms (median of `reps`)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    alm = pf.zeros_alm(plan.lmax, plan.ntrans, device=dev)
    alm.real.normal_()
    f = pf.zeros_field(plan.npts, plan.ntrans, device=dev)
    f.real.normal_()
    a2 = pf.zeros_alm(plan.lmax, plan.ntrans, device=dev)
    f2 = pf.zeros_field(plan.npts, plan.ntrans, device=dev)
    for _ in range(warmup):
        plan.mul(f2, alm)
        plan.mul_adjoint(a2, f)
    times = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.mul(f2, alm)
        plan.mul_adjoint(a2, f)
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    times.sort()
    return times[len(times) // 2]


def tune(theta, phi, *, lmax, tol=1e-10, ntrans=1, precision="fp64", cache=None,
         retune=False, **plan_kwargs) -> dict:
    """Tuned shape keyword arguments for Plan(theta, phi, lmax=..., ...)."""
    from . import Plan  # noqa: the package's Plan
    import importlib
    pf = importlib.import_module(__package__)
    path = cache or default_cache_path()
    key = shape_class(lmax, len(theta), tol, ntrans, precision)
    with _lock:
        table = _load(path)
    if not retune and key in table:
        return dict(table[key]["shapes"])
    best = {}
    best_ms = None
    base = dict(lmax=lmax, tol=tol, ntrans=ntrans, precision=precision, **plan_kwargs)
    for name, values in CANDIDATES:
        for v in values:
            trial = dict(best)
            trial[name] = v
            if best_ms is not None and trial == best:
                continue
            plan = Plan(theta, phi, **base, **trial)
            ms = time_plan(pf, plan)
            del plan
            if best_ms is None or ms < best_ms:
                best, best_ms = trial, ms
    best = {k: v for k, v in best.items() if v != 0}
    with _lock:
        table = _load(path)
        table[key] = {"shapes": best, "ms": best_ms}
        _store(path, table)
    return best


def tuned_plan(theta, phi, *, lmax, tol=1e-10, ntrans=1, precision="fp64", cache=None,
               **plan_kwargs):
    """Plan(...) built with the tuned tile shapes of its shape class (tuning it if needed)."""
    from . import Plan
    shapes = tune(theta, phi, lmax=lmax, tol=tol, ntrans=ntrans, precision=precision,
                  cache=cache, **plan_kwargs)
    return Plan(theta, phi, lmax=lmax, tol=tol, ntrans=ntrans, precision=precision,
                **plan_kwargs, **shapes)
