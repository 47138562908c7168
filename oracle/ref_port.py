"""CPU port of the reference PSTM kernel, FP32 torch.  TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline / reference arm
of ``bench.py`` may import this module.

It restates the algorithm of the reference's ``migrate_kirchhoff_full``
(processors/migration/kirchhoff_kernel.py:459-854) with the same float32 torch
arithmetic, so that it can stand in for the reference where the reference
itself is not installed (it is a Python package that does not travel):

* output points are processed in tiles of 100 (il-major order, :519-530);
* per tile, traces whose midpoint lies within A + tile_radius + 100 m of the
  tile centre are kept (:572-602);
* per tile, the horizontal leg distances and the constant per-leg aperture
  mask are formed once (:611-635);
* depths are processed in batches sized for ~500 MB of temporaries
  (:642-646); per depth, the clamped sample index, floor/ceil gathers, linear
  blend, weighted sum and fold are formed and written to the image (:700-730).

The arithmetic is expressed in this file's own code.  Golden fixtures made by
running the reference itself (tests/golden/make_golden.py) pin it.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np
import torch


def migrate_full_port(traces: torch.Tensor, source_x: torch.Tensor, source_y: torch.Tensor,
                      receiver_x: torch.Tensor, receiver_y: torch.Tensor, output_x: torch.Tensor,
                      output_y: torch.Tensor, depth_axis: torch.Tensor, velocity: float,
                      dt_ms: float, t_min_ms: float, max_aperture_m: float, max_angle_deg: float,
                      n_il: int, n_xl: int, use_time_dependent_aperture: bool = False,
                      tile: int = 100, column_subset: Optional[np.ndarray] = None):
    """Returns (image, fold) as (n_depths, n_il, n_xl) float32 tensors.

    ``column_subset`` (sorted flat column indices) restricts the work to those
    output points; used to time a bounded sample of a large configuration.
    """
    n_s, n_tr = traces.shape
    n_d = depth_axis.shape[0]
    n_out = n_il * n_xl
    image = torch.zeros(n_d, n_out, dtype=torch.float32)
    fold = torch.zeros(n_d, n_out, dtype=torch.float32)
    theta = math.radians(max_angle_deg)
    tan_theta = math.tan(theta)
    k_time = 1000.0 / velocity
    mid_x = (source_x + receiver_x) / 2
    mid_y = (source_y + receiver_y) / 2
    pts = np.arange(n_out) if column_subset is None else np.asarray(column_subset)
    for start in range(0, pts.shape[0], tile):
        sel = torch.from_numpy(pts[start:start + tile].astype(np.int64))
        px = output_x[sel]
        py = output_y[sel]
        cx = (px.min() + px.max()) / 2
        cy = (py.min() + py.max()) / 2
        rad = torch.sqrt(((px - cx) ** 2 + (py - cy) ** 2).max())
        near = torch.sqrt((mid_x - cx) ** 2 + (mid_y - cy) ** 2) < (max_aperture_m + rad + 100)
        cand = torch.nonzero(near).flatten()
        nf = cand.numel()
        if nf == 0:
            continue
        sxf, syf = source_x[cand], source_y[cand]
        rxf, ryf = receiver_x[cand], receiver_y[cand]
        data = traces[:, cand]
        hs2 = (px[:, None] - sxf[None, :]) ** 2 + (py[:, None] - syf[None, :]) ** 2
        hr2 = (px[:, None] - rxf[None, :]) ** 2 + (py[:, None] - ryf[None, :]) ** 2
        hs = torch.sqrt(hs2)
        hr = torch.sqrt(hr2)
        ap_const = (hs < max_aperture_m) & (hr < max_aperture_m)
        npt = px.shape[0]
        per_depth = npt * nf * 4 * 8
        batch = max(1, min(50, int(500_000_000 / max(per_depth, 1))))
        col = torch.arange(nf).unsqueeze(0).expand(npt, -1).reshape(-1)
        for d0 in range(0, n_d, batch):
            d1 = min(n_d, d0 + batch)
            z = depth_axis[d0:d1].view(-1, 1, 1)
            rs = torch.sqrt(hs2.unsqueeze(0) + z ** 2)
            rr = torch.sqrt(hr2.unsqueeze(0) + z ** 2)
            ang_s = torch.atan2(hs.unsqueeze(0), z + 1e-6)
            ang_r = torch.atan2(hr.unsqueeze(0), z + 1e-6)
            if use_time_dependent_aperture:
                apz = torch.clamp(depth_axis[d0:d1] * tan_theta, max=max_aperture_m).view(-1, 1, 1)
                ap = (hs.unsqueeze(0) < apz) & (hr.unsqueeze(0) < apz)
            else:
                ap = ap_const.unsqueeze(0).expand(d1 - d0, -1, -1)
            ok = ap & (ang_s < theta) & (ang_r < theta)
            tt = (rs + rr) * k_time
            w = (z / (rs + 1e-6)) * (z / (rr + 1e-6)) / (rs * rr + 1e-6)
            for q in range(d1 - d0):
                si = torch.clamp((tt[q] - t_min_ms) / dt_ms, 0, n_s - 1.001)
                lo = si.long()
                hi = (lo + 1).clamp(max=n_s - 1)
                fr = si - lo.float()
                a0 = data[lo.reshape(-1), col].reshape(npt, nf)
                a1 = data[hi.reshape(-1), col].reshape(npt, nf)
                okf = ok[q].float()
                image[d0 + q, sel] = ((a0 + fr * (a1 - a0)) * w[q] * okf).sum(dim=1)
                fold[d0 + q, sel] = okf.sum(dim=1)
    return image.view(n_d, n_il, n_xl), fold.view(n_d, n_il, n_xl)


def engine_full_port(traces: np.ndarray, source_x, source_y, receiver_x, receiver_y, origin_x,
                     origin_y, il_spacing, xl_spacing, n_il, n_xl, dt_ms, t_min_ms, n_times=None,
                     velocity_mps=2500.0, max_aperture_m=5000.0, max_angle_deg=60.0,
                     use_time_dependent_aperture=False, column_subset=None):
    """Restates MigrationEngine.migrate_bin_full's set-up (migration_engine.py:284-339):
    float32 inputs, grid x = origin_x + il*dx, y = origin_y + xl*dy (azimuth
    ignored), z = V t / 2; no fold normalisation (callers apply it)."""
    n_s = traces.shape[0]
    n_t = n_times if n_times is not None else n_s
    tr = torch.from_numpy(np.ascontiguousarray(traces, dtype=np.float32))
    f32 = lambda a: torch.from_numpy(np.asarray(a, dtype=np.float32))
    il = torch.arange(n_il, dtype=torch.float32) * il_spacing + origin_x
    xl = torch.arange(n_xl, dtype=torch.float32) * xl_spacing + origin_y
    gx, gi = torch.meshgrid(xl, il, indexing="xy")
    out_x = gi.flatten()
    out_y = gx.flatten()
    t_ms = torch.arange(n_t, dtype=torch.float32) * dt_ms + t_min_ms
    depth = velocity_mps * (t_ms / 1000.0) / 2.0
    return migrate_full_port(tr, f32(source_x), f32(source_y), f32(receiver_x), f32(receiver_y),
                             out_x, out_y, depth, velocity_mps, dt_ms, t_min_ms, max_aperture_m,
                             max_angle_deg, n_il, n_xl, use_time_dependent_aperture,
                             column_subset=column_subset)
