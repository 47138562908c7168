"""The reference's time-domain RMS operator on the CUDA kernel.

``migrate_kirchhoff_time_domain_rms`` keeps the signature and results of
processors/migration/kirchhoff_kernel.py:1313-1783 (and
``MigrationEngine.migrate_bin_time_domain_rms`` those of
migration_engine.py:633-802).  It is a different operator from the Kirchhoff
summation the rest of this package implements: each input sample of a trace is
moved to t_out = sqrt(t_in^2 + 4 h_eff^2 / V_rms(t_in)^2), h being the distance
from the trace's midpoint to an output point, and added into the trace's OWN
midpoint column, once for every output point of every tile whose trace list
holds the trace.

Host side (this module, device tensor operations in float32, in the
reference's order so every rounding is the reference's):
* trace midpoints, half-offsets and midpoint columns (:1412-1437);
* the tile size the reference shrinks to under its memory target (:1463-1472);
* per tile of consecutive output points: the traces within aperture + tile
  radius + 100 m of the tile centre, the nearest ``max_traces_per_tile`` kept
  (:1539-1568) -- the (tile, trace) pairs;
* V_rms at the input times (:1474-1488).
The pairs are sorted by the trace's column and handed to
``pstm_time_rms_migrate``, whose kernel owns one column per CTA.

``use_half_precision`` is accepted and ignored, as in the reference (float16
overflows there, :1386-1395).  Exact distance ties at the trace cap are
resolved by ``torch.topk``; the reference's ``torch.argsort`` is not stable
either, so which of two equidistant traces is kept is unspecified in both.
"""
from __future__ import annotations

import ctypes as C
import logging
import time
from typing import Callable, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .kernel_backend import require_cuda
from .kirchhoff import _ptr, _stream_handle

logger = logging.getLogger(__name__)


def effective_tile_size(tile_size: int, max_traces_per_tile: int, sample_batch_size: int) -> int:
    """The reference's tile after its 12 GB tensor-memory bound (:1463-1472)."""
    max_elements = int(12.0 * 1024 ** 3 // (4 * 10))
    cap = max(50, max_elements // max(1, max_traces_per_tile * sample_batch_size))
    return min(int(tile_size), cap)


def _scalar(x: float, like: torch.Tensor) -> torch.Tensor:
    """x as a 0-d float32 tensor on ``like``'s device.  Dividing a CUDA tensor
    by a Python number multiplies by its float32 reciprocal, which rounds
    differently from the reference's division; dividing by a tensor divides."""
    return torch.tensor(x, dtype=like.dtype, device=like.device)


def trace_geometry(source_x, source_y, receiver_x, receiver_y, origin_x, origin_y,
                   il_spacing, xl_spacing, azimuth_deg, n_il, n_xl):
    """Midpoints, squared half-offsets and the midpoint column il * n_xl + xl
    (truncated toward zero, clamped to the grid), float32 as :1412-1437."""
    mid_x = (source_x + receiver_x) / 2.0
    mid_y = (source_y + receiver_y) / 2.0
    hx = (receiver_x - source_x) / 2.0
    hy = (receiver_y - source_y) / 2.0
    hoff_sq = hx ** 2 + hy ** 2
    cos_az = np.cos(np.radians(azimuth_deg))
    sin_az = np.sin(np.radians(azimuth_deg))
    dx = mid_x - origin_x
    dy = mid_y - origin_y
    il = (dx * cos_az + dy * sin_az) / _scalar(il_spacing, dx)
    xl = (-dx * sin_az + dy * cos_az) / _scalar(xl_spacing, dx)
    col = il.long().clamp(0, n_il - 1) * n_xl + xl.long().clamp(0, n_xl - 1)
    return mid_x, mid_y, hoff_sq, col


def tile_pairs(output_x: torch.Tensor, output_y: torch.Tensor, mid_x: torch.Tensor,
               mid_y: torch.Tensor, tile: int, max_aperture_m: float,
               max_traces_per_tile: int, elements: int = 1 << 26):
    """(tile, trace) int64 pairs of the reference's per-tile trace selection
    (:1539-1568), tiles in order and traces ascending within a tile.  Tiles
    are processed in chunks of about ``elements`` (tile, trace) distances."""
    n_out = output_x.numel()
    n_tr = mid_x.numel()
    dev = output_x.device
    n_tiles = (n_out + tile - 1) // tile
    empty = torch.empty(0, dtype=torch.int64, device=dev)
    if n_tr == 0 or n_tiles == 0:
        return empty, empty
    pad = n_tiles * tile - n_out
    # repeating the last point changes no tile's min, max or radius
    ox = torch.cat([output_x, output_x[-1:].expand(pad)]).view(n_tiles, tile)
    oy = torch.cat([output_y, output_y[-1:].expand(pad)]).view(n_tiles, tile)
    cx = (ox.min(1).values + ox.max(1).values) / 2
    cy = (oy.min(1).values + oy.max(1).values) / 2
    rad = torch.sqrt(((ox - cx[:, None]) ** 2 + (oy - cy[:, None]) ** 2).max(1).values)
    thr = max_aperture_m + rad + 100
    tiles, traces = [], []
    step = max(1, elements // max(n_tr, 1))
    for a in range(0, n_tiles, step):
        b = min(a + step, n_tiles)
        dist = torch.sqrt((mid_x[None, :] - cx[a:b, None]) ** 2
                          + (mid_y[None, :] - cy[a:b, None]) ** 2)
        sel = dist < thr[a:b, None]
        over = torch.nonzero(sel.sum(1) > max_traces_per_tile).flatten()
        if over.numel():
            d = dist[over].masked_fill(~sel[over], float("inf"))
            keep = torch.topk(d, max_traces_per_tile, dim=1, largest=False).indices
            m = torch.zeros_like(sel[over])
            m.scatter_(1, keep, True)
            sel[over] = m
        nz = torch.nonzero(sel)
        tiles.append(nz[:, 0] + a)
        traces.append(nz[:, 1])
    return torch.cat(tiles), torch.cat(traces)


def column_pairs(output_x: torch.Tensor, output_y: torch.Tensor, mid_x: torch.Tensor,
                 mid_y: torch.Tensor, col: torch.Tensor, tile: int, max_aperture_m: float,
                 max_traces_per_tile: int):
    """The (tile, trace) pairs in the form ``pstm_time_rms_migrate`` takes them:
    sorted by the trace's midpoint column (stable, so tile order is kept within
    a column), as (pair_trace int32, pair_tile int32, seg_off int64 with one
    more entry than there are columns with pairs, seg_col int32)."""
    p_tile, p_trace = tile_pairs(output_x, output_y, mid_x, mid_y, tile, max_aperture_m,
                                 max_traces_per_tile)
    key, order = torch.sort(col[p_trace], stable=True)
    pair_trace = p_trace[order].to(torch.int32).contiguous()
    pair_tile = p_tile[order].to(torch.int32).contiguous()
    seg_col, counts = torch.unique_consecutive(key, return_counts=True)
    seg_off = torch.zeros(seg_col.numel() + 1, dtype=torch.int64, device=key.device)
    torch.cumsum(counts, 0, out=seg_off[1:])
    return pair_trace, pair_tile, seg_off, seg_col.to(torch.int32).contiguous()


def launch_time_rms(traces: torch.Tensor, mid_x: torch.Tensor, mid_y: torch.Tensor,
                    hoff_sq: torch.Tensor, output_x: torch.Tensor, output_y: torch.Tensor,
                    v_rms: torch.Tensor, pairs, tile: int, dt_ms: float, t_min_ms: float,
                    max_aperture_m: float, max_angle_deg: float,
                    use_time_dependent_aperture: bool, image: torch.Tensor,
                    fold: torch.Tensor) -> None:
    """One ``pstm_time_rms_migrate`` launch on the current stream: ``traces``
    (n_samples, n_traces) float32, the per-trace and per-point float32 arrays,
    V_rms per input sample, ``pairs`` from ``column_pairs``; image and fold
    (n_times, n_points) float32 contiguous, overwritten."""
    n_s, n_tr = traces.shape
    pair_trace, pair_tile, seg_off, seg_col = pairs
    p = _lib.TimeRmsParams(n_samples=n_s, n_traces=n_tr, n_points=output_x.numel(),
                           n_times=image.shape[0], tile=tile, dt_ms=float(dt_ms),
                           t_min_ms=float(t_min_ms), max_aperture_m=float(max_aperture_m),
                           max_angle_deg=float(max_angle_deg),
                           time_dependent_aperture=1 if use_time_dependent_aperture else 0)
    args = [a.contiguous() for a in (traces, mid_x, mid_y, hoff_sq, output_x, output_y, v_rms)]
    _lib.check(_lib.lib().pstm_time_rms_migrate(
        C.byref(p), *(_ptr(a) for a in args), _ptr(pair_trace), _ptr(pair_tile),
        int(pair_trace.numel()), _ptr(seg_off), _ptr(seg_col), int(seg_col.numel()),
        _ptr(image), _ptr(fold), _stream_handle()))


def migrate_kirchhoff_time_domain_rms(
    traces: torch.Tensor,
    source_x: torch.Tensor,
    source_y: torch.Tensor,
    receiver_x: torch.Tensor,
    receiver_y: torch.Tensor,
    output_x: torch.Tensor,
    output_y: torch.Tensor,
    time_axis_ms: torch.Tensor,
    velocity_model,
    dt_ms: float,
    t_min_ms: float,
    max_aperture_m: float,
    max_angle_deg: float,
    n_il: int,
    n_xl: int,
    origin_x: float,
    origin_y: float,
    il_spacing: float,
    xl_spacing: float,
    azimuth_deg: float,
    tile_size: int = 100,
    sample_batch_size: int = 200,
    max_traces_per_tile: int = 5000,
    progress_callback: Optional[Callable[[float, str], None]] = None,
    enable_profiling: bool = False,
    use_time_dependent_aperture: bool = True,
    use_half_precision: bool = True,
) -> Tuple[torch.Tensor, torch.Tensor]:
    """(image, fold), each (n_times, n_il, n_xl) float32 on the traces' device.

    ``traces`` (n_samples, n_traces), input sample i at time i * dt_ms;
    ``velocity_model`` any object with ``rms_velocity_at_time`` (the
    engine's ``VelocityModel``); output time k at t_min_ms + k * dt_ms for
    k < len(time_axis_ms)."""
    require_cuda()
    dev = traces.device
    if dev.type != "cuda":
        raise ValueError("migrate_kirchhoff_time_domain_rms runs on a CUDA device only")
    t0 = time.time()
    f32 = torch.float32
    tr = traces.to(dev, f32).contiguous()
    n_s, n_tr = tr.shape
    n_times = int(time_axis_ms.shape[0])
    n_out = n_il * n_xl
    if output_x.numel() != n_out or output_y.numel() != n_out:
        raise ValueError("output_x/output_y must hold n_il * n_xl points")
    if n_tr >= 2 ** 31 or n_out >= 2 ** 31:
        raise ValueError("more than 2^31 - 1 traces or output points")
    sx, sy, rx, ry = (a.to(dev, f32) for a in (source_x, source_y, receiver_x, receiver_y))
    ox, oy = output_x.to(dev, f32).contiguous(), output_y.to(dev, f32).contiguous()
    if progress_callback:
        progress_callback(0.0, "Starting time-domain (RMS) migration")

    mid_x, mid_y, hoff_sq, col = trace_geometry(sx, sy, rx, ry, origin_x, origin_y, il_spacing,
                                                xl_spacing, azimuth_deg, n_il, n_xl)
    tile = effective_tile_size(tile_size, max_traces_per_tile, sample_batch_size)
    t_in = 0.0 + torch.arange(n_s, device=dev, dtype=f32) * dt_ms
    v = velocity_model.rms_velocity_at_time(t_in)
    v = (v if isinstance(v, torch.Tensor) else torch.as_tensor(np.asarray(v))).to(dev, f32)
    v = v.expand(n_s).contiguous()

    pairs = column_pairs(ox, oy, mid_x, mid_y, col, tile, max_aperture_m, max_traces_per_tile)
    image = torch.empty((n_times, n_il, n_xl), dtype=f32, device=dev)
    fold = torch.empty_like(image)
    with torch.cuda.device(dev):
        launch_time_rms(tr, mid_x, mid_y, hoff_sq, ox, oy, v, pairs, tile, dt_ms, t_min_ms,
                        max_aperture_m, max_angle_deg, use_time_dependent_aperture, image, fold)
    pair_trace, seg_col = pairs[0], pairs[3]
    if enable_profiling:
        torch.cuda.synchronize(dev)
        logger.info("time-domain (RMS): %d tiles of %d points, %d (tile, trace) pairs, "
                    "%d columns, %.3f s", (n_out + tile - 1) // tile, tile,
                    pair_trace.numel(), seg_col.numel(), time.time() - t0)
    if progress_callback:
        progress_callback(1.0, "Time-domain (RMS) migration complete")
    return image, fold
