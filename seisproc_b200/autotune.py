"""Kernel-shape autotuner.

A kernel shape fixes the output tile (columns per CTA, tile_il x tile_xl) and
the time window per CTA (warps per column x 64 x groups per lane).  For a
given problem the tuner builds a plan per candidate shape, times the forward
migration with CUDA events (after a warm-up), and keeps the fastest.  Results
are cached per problem class -- (grid kind, n_times bucket, n_samples bucket,
traces-per-column bucket, storage) -- in a JSON file, so later plans pick the
shape without timing.
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Callable, Dict, Iterable, Optional, Tuple

import torch

# shape id -> (columns, tile_il, tile_xl, samples per CTA window)
SHAPES: Dict[int, Tuple[int, int, int, int]] = {
    1: (8, 2, 4, 1024),
    2: (4, 2, 2, 1024),
    3: (16, 4, 4, 512),
    4: (4, 2, 2, 512),
    5: (8, 8, 1, 1024),
    6: (4, 4, 1, 512),
    7: (2, 2, 1, 512),
    8: (4, 4, 1, 1024),
    9: (16, 16, 1, 512),
}
LINE_SHAPES = (5, 6, 7, 8, 9)
GRID_SHAPES = (1, 2, 3, 4)

_CACHE_PATH = os.environ.get("SEISPSTM_TUNE_CACHE",
                             os.path.join(os.path.expanduser("~"), ".cache", "seispstm_tune.json"))
_lock = threading.Lock()


def _bucket(v: float) -> int:
    return int(round(math.log2(max(v, 1.0))))


def problem_key(n_xl: int, n_times: int, n_samples: int, traces_per_column: float,
                storage: str) -> str:
    kind = "line" if n_xl < 2 else "grid"
    return f"{kind}/t{_bucket(n_times)}/s{_bucket(n_samples)}/c{_bucket(traces_per_column)}/{storage}"


def candidates(n_xl: int) -> Iterable[int]:
    return LINE_SHAPES if n_xl < 2 else GRID_SHAPES


def _load() -> dict:
    try:
        with open(_CACHE_PATH) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(d: dict) -> None:
    try:
        os.makedirs(os.path.dirname(_CACHE_PATH), exist_ok=True)
        tmp = _CACHE_PATH + ".tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, _CACHE_PATH)
    except Exception:
        pass


def cached_variant(key: str) -> Optional[int]:
    with _lock:
        v = _load().get(key)
    return int(v["variant"]) if v else None


def tune(make_plan: Callable[[int], "object"], traces: torch.Tensor, velocity, key: str,
         variants: Iterable[int], repeats: int = 2, force: bool = False) -> Tuple[int, dict]:
    """Time each candidate shape; returns (best variant, {variant: ms}).

    ``make_plan(variant)`` must return a PSTMPlan for the problem."""
    if not force:
        v = cached_variant(key)
        if v is not None:
            return v, {}
    times = {}
    for var in variants:
        plan = make_plan(var)
        try:
            plan.load_traces(traces)
            plan.migrate_loaded(velocity, with_fold=False)  # warm-up
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(repeats):
                plan.migrate_loaded(velocity, with_fold=False)
            b.record()
            torch.cuda.synchronize()
            plan.check()
            times[var] = a.elapsed_time(b) / repeats
        finally:
            plan.close()
    best = min(times, key=times.get)
    with _lock:
        d = _load()
        d[key] = {"variant": best, "ms": times}
        _store(d)
    return best, times
