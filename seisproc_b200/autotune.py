"""Kernel-shape autotuner.

A kernel shape fixes the output tile (columns per CTA, tile_il x tile_xl) and
the time window per CTA (warps per column x 64 x groups per lane): 1024, 512,
256 or 128 output samples.  Shapes of 256 threads run two CTAs per SM, each
with half the shared memory.  For a problem the tuner builds a plan per candidate
shape on a centred crop of the output grid (at most 32 x 32 columns, all output
times, the traces within reach of the crop), times the forward migration with
CUDA events and keeps the fastest.  The kernel's run time depends on the
geometry, the grid and the storage, not on the sample values, so the crop is
migrated with zero-valued traces and no trace data is needed.

Results are cached per problem class -- (grid kind, n_times bucket, n_samples
bucket, traces-per-column bucket, storage) -- under the device name and the
library's ABI version, in a JSON file (``SEISPSTM_TUNE_CACHE``, default
``~/.cache/seispstm_tune.json``), so a cache written on another GPU or by
another build of the library is never used.  ``choose_variant`` is what the
engine, the migrator and the batched launch call for plans built with
``variant=0``: a cached shape, else a tuning run (``tune_on_crop``), else the
built-in heuristic.
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Callable, Dict, Iterable, Optional, Sequence, Tuple

import numpy as np
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
    10: (16, 4, 4, 256),
    11: (16, 4, 4, 128),
    12: (16, 16, 1, 256),
    13: (8, 2, 4, 512),
}
LINE_SHAPES = (5, 6, 7, 8, 9, 12)
GRID_SHAPES = (1, 2, 3, 4, 10, 11, 13)
CROP = 32  # columns per crop side

_lock = threading.Lock()


def cache_path() -> str:
    return os.environ.get("SEISPSTM_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "seispstm_tune.json"))


def _bucket(v: float) -> int:
    return int(round(math.log2(max(v, 1.0))))


def device_tag(device=None) -> str:
    """Device name and library ABI version: the scope of a cached result."""
    from . import _lib
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    return f"{torch.cuda.get_device_name(dev)}/abi{_lib.lib().pstm_abi_version()}"


def problem_key(n_xl: int, n_times: int, n_samples: int, traces_per_column: float,
                storage: str) -> str:
    kind = "line" if n_xl < 2 else "grid"
    return f"{kind}/t{_bucket(n_times)}/s{_bucket(n_samples)}/c{_bucket(traces_per_column)}/{storage}"


def candidates(n_xl: int) -> Iterable[int]:
    return LINE_SHAPES if n_xl < 2 else GRID_SHAPES


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except Exception:
        return {}


def _store(d: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except Exception:
        pass


def cached_variant(key: str, device=None) -> Optional[int]:
    tag = device_tag(device)
    with _lock:
        v = _load().get(tag, {}).get(key)
    return int(v["variant"]) if v else None


def record(key: str, best: int, times: Dict[int, float], device=None) -> None:
    tag = device_tag(device)
    with _lock:
        d = _load()
        d.setdefault(tag, {})[key] = {"variant": int(best),
                                      "ms": {str(k): float(v) for k, v in times.items()}}
        _store(d)


def tune(make_plan: Callable[[int], "object"], traces: torch.Tensor, velocity, key: str,
         variants: Iterable[int], repeats: int = 2, force: bool = False,
         device=None) -> Tuple[int, dict]:
    """Time each candidate shape; returns (best variant, {variant: ms}) and
    records the winner.  ``make_plan(variant)`` must return a PSTMPlan for the
    problem; ``traces`` are loaded into it.  A cached result is returned
    without timing (empty times) unless ``force``."""
    if not force:
        v = cached_variant(key, device)
        if v is not None:
            return v, {}
    times = {}
    for var in variants:
        try:
            plan = make_plan(var)
        except (ValueError, NotImplementedError):
            continue  # e.g. traces too long for this shape's shared-memory ring
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
    record(key, best, times, device)
    return best, times


def _crop(coords: Sequence[torch.Tensor], n_il: int, n_xl: int, origin_x: float,
          origin_y: float, il_dx: float, il_dy: float, xl_dx: float, xl_dy: float,
          aperture: float):
    """The centred crop of at most CROP x CROP columns: its first column's
    (il, xl), size, origin, and the indices of the traces with both legs
    within the aperture of some crop column."""
    c_il, c_xl = min(CROP, n_il), min(CROP, n_xl)
    i0, j0 = (n_il - c_il) // 2, (n_xl - c_xl) // 2
    ox = origin_x + i0 * il_dx + j0 * xl_dx
    oy = origin_y + i0 * il_dy + j0 * xl_dy
    ei, ej = 0.5 * (c_il - 1), 0.5 * (c_xl - 1)
    cx, cy = ox + ei * il_dx + ej * xl_dx, oy + ei * il_dy + ej * xl_dy
    rad = max(math.hypot(a * il_dx + b * xl_dx, a * il_dy + b * xl_dy)
              for a in (-ei, ei) for b in (-ej, ej))
    reach = aperture + rad + 1.0
    sx, sy, rx, ry = (c.to(torch.float64) for c in coords)
    keep = ((torch.hypot(sx - cx, sy - cy) <= reach) & (torch.hypot(rx - cx, ry - cy) <= reach))
    idx = torch.nonzero(keep).flatten()
    return i0, j0, c_il, c_xl, ox, oy, idx, reach


def choose_variant(coords: Sequence[torch.Tensor], *, n_il: int, n_xl: int, n_times: int,
                   origin_x: float, origin_y: float, il_dx: float, il_dy: float, xl_dx: float,
                   xl_dy: float, n_samples: int, max_aperture_m: float, velocity: torch.Tensor,
                   storage: str = "f32", antialias: bool = False, tune_on_miss: bool = True,
                   **plan_kw) -> int:
    """Kernel shape for a problem: the cached winner of its class, else (with
    ``tune_on_miss``) the winner of a timing run on the centred crop, else 0
    (the library's heuristic).  ``coords`` are the device tensors (sx, sy, rx,
    ry); ``velocity`` is V_rms on the device (constant, (n_times,) or one value
    per output sample); ``plan_kw`` are the remaining PSTMPlan arguments."""
    from .kirchhoff import PSTMPlan
    if plan_kw.get("taper_width", 0.0) > 0 or plan_kw.get("ray_gradient", 0.0) != 0:
        return 0  # the tapered and curved-ray kernels exist for one shape each
    i0, j0, c_il, c_xl, ox, oy, idx, reach = _crop(coords, n_il, n_xl, origin_x, origin_y,
                                                   il_dx, il_dy, xl_dx, xl_dy, max_aperture_m)
    n_sel = int(idx.numel())
    if n_sel == 0:
        return 0
    tpc = n_sel * (max_aperture_m / reach) ** 2  # traces within one column's aperture
    key = problem_key(n_xl, n_times, n_samples, tpc, storage + ("/aa" if antialias else ""))
    dev = coords[0].device
    v = cached_variant(key, dev)
    if v is not None or not tune_on_miss:
        return v or 0
    vel = velocity
    if vel.numel() == n_times * n_il * n_xl:
        vel = vel.reshape(n_times, n_il, n_xl)[:, i0:i0 + c_il, j0:j0 + c_xl].contiguous()
    sub = [c.index_select(0, idx).contiguous() for c in coords]
    zeros = torch.zeros((n_samples, n_sel), device=dev)
    kw = dict(plan_kw, n_il=c_il, n_xl=c_xl, n_times=n_times, origin_x=ox, origin_y=oy,
              il_dx=il_dx, il_dy=il_dy, xl_dx=xl_dx, xl_dy=xl_dy, n_samples=n_samples,
              max_aperture_m=max_aperture_m, storage=storage, antialias=antialias)
    best, _ = tune(lambda var: PSTMPlan(*sub, variant=var, **kw), zeros, vel, key,
                   candidates(n_xl), force=True, device=dev)
    return best
