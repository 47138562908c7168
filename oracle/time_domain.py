"""Oracle for the time-domain RMS operator: a float32 numpy restatement.

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` may import this module, as the
checker of the CUDA path; nothing in the package calls it.

The reference's ``migrate_kirchhoff_time_domain_rms``
(processors/migration/kirchhoff_kernel.py:1313-1783), called from
``MigrationEngine.migrate_bin_time_domain_rms``
(processors/migration/migration_engine.py:633-802), maps each input sample of
each trace to an output time t_out = sqrt(t_in^2 + 4 h_eff^2 / V_rms(t_in)^2)
and scatters it, weighted, into the trace's OWN midpoint column -- once per
output point of every tile whose trace list holds the trace.  Its output time
index is a truncation of a float32 expression, so a float64 restatement would
move contributions across sample boundaries; this oracle therefore repeats the
reference's float32 operations in the reference's order (every Python scalar
is rounded to float32 first, as torch does), which makes the output indices
bit-identical, and accumulates the sums in float64.

Square roots here are IEEE (numpy's, as on a GPU); the reference's CPU run
takes torch's CPU float32 sqrt, which is an ulp off on about 0.7 % of inputs,
so where such an ulp straddles an integer output index the reference puts
the contribution one sample over (a few dozen of 4e7 fold counts on a
3000-trace case).  ``time_domain_rms_torch_port`` below repeats the reference
with torch itself and is bit-identical to it.  The angle mask uses
``np.arctan2`` where the reference uses torch's; they differ by an ulp on many
inputs but moved no contribution in the cases measured.  Pinned by golden
vectors made by running the reference (tests/golden/make_time_domain_golden.py).
"""
from __future__ import annotations

import numpy as np

f32 = np.float32


def output_grid_f32(origin_x, origin_y, il_spacing, xl_spacing, azimuth_deg, n_il, n_xl):
    """Output point coordinates, flattened il-major (migration_engine.py:727-737)."""
    cos_az, sin_az = f32(np.cos(np.radians(azimuth_deg))), f32(np.sin(np.radians(azimuth_deg)))
    il = np.arange(n_il, dtype=f32) * f32(il_spacing)
    xl = np.arange(n_xl, dtype=f32) * f32(xl_spacing)
    il_g = np.repeat(il, n_xl)
    xl_g = np.tile(xl, n_il)
    ox = f32(origin_x) + il_g * cos_az - xl_g * sin_az
    oy = f32(origin_y) + il_g * sin_az + xl_g * cos_az
    return ox.astype(f32), oy.astype(f32)


def effective_tile_size(tile_size, max_traces_per_tile, sample_batch_size):
    """kirchhoff_kernel.py:1463-1472: the tile shrinks to bound tensor memory."""
    max_elements = int(12.0 * 1024 ** 3 // (4 * 10))
    cap = max(50, max_elements // max(1, max_traces_per_tile * sample_batch_size))
    return min(tile_size, cap)


def trace_columns_f32(mid_x, mid_y, origin_x, origin_y, il_spacing, xl_spacing, azimuth_deg,
                      n_il, n_xl):
    """Each trace's midpoint bin (kirchhoff_kernel.py:1420-1437): rotate,
    divide by the spacing, truncate toward zero, clamp to the grid."""
    cos_az, sin_az = f32(np.cos(np.radians(azimuth_deg))), f32(np.sin(np.radians(azimuth_deg)))
    dx = mid_x - f32(origin_x)
    dy = mid_y - f32(origin_y)
    il = (dx * cos_az + dy * sin_az) / f32(il_spacing)
    xl = (-dx * sin_az + dy * cos_az) / f32(xl_spacing)
    il_i = np.clip(np.trunc(il).astype(np.int64), 0, n_il - 1)
    xl_i = np.clip(np.trunc(xl).astype(np.int64), 0, n_xl - 1)
    return il_i, xl_i


def tile_trace_lists(output_x, output_y, mid_x, mid_y, tile, aperture, cap):
    """Per tile of ``tile`` consecutive output points: the traces whose
    midpoint is within aperture + tile radius + 100 m of the tile centre,
    keeping the ``cap`` nearest (kirchhoff_kernel.py:1543-1568).  Exact
    distance ties at the cap are broken by trace order here; the reference's
    unstable argsort leaves them unspecified."""
    out = []
    for s in range(0, output_x.size, tile):
        tx, ty = output_x[s:s + tile], output_y[s:s + tile]
        cx = (tx.min() + tx.max()) / f32(2)
        cy = (ty.min() + ty.max()) / f32(2)
        rad = np.sqrt(((tx - cx) ** 2 + (ty - cy) ** 2).max())
        dist = np.sqrt((mid_x - cx) ** 2 + (mid_y - cy) ** 2)
        sel = np.nonzero(dist < (f32(aperture) + rad + f32(100)))[0]
        if sel.size > cap:
            sel = sel[np.argsort(dist[sel], kind="stable")[:cap]]
        out.append((s, min(s + tile, output_x.size), sel))
    return out


def time_domain_rms_f32(traces, source_x, source_y, receiver_x, receiver_y, v_rms_in,
                        origin_x, origin_y, il_spacing, xl_spacing, azimuth_deg, n_il, n_xl,
                        dt_ms, t_min_ms, n_times, max_aperture_m, max_angle_deg,
                        tile_size=100, sample_batch_size=200, max_traces_per_tile=5000,
                        use_time_dependent_aperture=True, batch=64, tiles=None):
    """(image, fold) as float64 sums of the reference's float32 terms.

    ``traces`` (n_samples, n_traces) float32; ``v_rms_in`` the float32 V_rms at
    each INPUT time i * dt_ms (input traces start at t = 0,
    kirchhoff_kernel.py:1474-1484).  ``tiles``, a list of (first point, end
    point, trace indices), restricts the sum to those tiles (default: every
    tile, with the reference's trace lists)."""
    traces = np.asarray(traces, f32)
    n_s, n_tr = traces.shape
    sx, sy = np.asarray(source_x, f32), np.asarray(source_y, f32)
    rx, ry = np.asarray(receiver_x, f32), np.asarray(receiver_y, f32)
    mid_x, mid_y = (sx + rx) / f32(2), (sy + ry) / f32(2)
    hx, hy = (rx - sx) / f32(2), (ry - sy) / f32(2)
    hoff_sq = hx ** 2 + hy ** 2
    t_il, t_xl = trace_columns_f32(mid_x, mid_y, origin_x, origin_y, il_spacing, xl_spacing,
                                   azimuth_deg, n_il, n_xl)
    col = t_il * n_xl + t_xl
    ox, oy = output_grid_f32(origin_x, origin_y, il_spacing, xl_spacing, azimuth_deg, n_il, n_xl)
    tile = effective_tile_size(tile_size, max_traces_per_tile, sample_batch_size)

    theta = f32(np.radians(max_angle_deg))
    tan_t = f32(np.tan(np.radians(max_angle_deg)))
    A = f32(max_aperture_m)
    lim = f32(n_times - 0.001)
    t_in = np.arange(n_s, dtype=f32) * f32(dt_ms) + f32(0.0)
    t_in_sq = t_in ** 2
    v = np.asarray(v_rms_in, f32)
    v_sq = v ** 2
    n_cols = n_il * n_xl
    image = np.zeros(n_times * n_cols, np.float64)
    fold = np.zeros(n_times * n_cols, np.float64)

    if tiles is None:
        tiles = tile_trace_lists(ox, oy, mid_x, mid_y, tile, max_aperture_m,
                                 max_traces_per_tile)
    for p0, p1, sel in tiles:
        if sel.size == 0:
            continue
        dx = ox[p0:p1, None] - mid_x[None, sel]
        dy = oy[p0:p1, None] - mid_y[None, sel]
        h_sq = dx ** 2 + dy ** 2                       # (n_tile, n_sel)
        h = np.sqrt(h_sq)
        c = (f32(4.0) * (h_sq + hoff_sq[None, sel])) * f32(1e6)
        cols = np.broadcast_to(col[sel][None, :], h.shape)
        for b0 in range(0, n_s, batch):
            b1 = min(b0 + batch, n_s)
            vs = v_sq[b0:b1, None, None]
            vo = v[b0:b1, None, None]
            t_out = np.sqrt(t_in_sq[b0:b1, None, None] + c[None] / vs)
            idx = (t_out - f32(t_min_ms)) / f32(dt_ms)
            ok = (idx >= 0) & (idx < lim)
            if use_time_dependent_aperture:
                ap = np.minimum(t_out * vo / f32(2000.0) * tan_t, A)
                ok &= h[None] < ap
            else:
                ok &= h[None] < A
            z = vo * t_out / f32(2000.0)
            ok &= np.arctan2(np.broadcast_to(h[None], z.shape), z + f32(1e-6)) < theta
            r_sq = z ** 2 + h_sq[None]
            w = z / (np.sqrt(r_sq) * r_sq + f32(1e-10))
            amp = traces[b0:b1, sel][:, None, :] * w
            k = np.clip(np.trunc(idx).astype(np.int64), 0, n_times - 1)
            lin = k * n_cols + cols[None]
            np.add.at(image, lin[ok], amp[ok].astype(np.float64))
            np.add.at(fold, lin[ok], 1.0)
    shape = (n_times, n_il, n_xl)
    return image.reshape(shape), fold.reshape(shape)


def rms_velocity_torch_order_f32(velocity_type, v0, gradient, t_ms):
    """V_rms(t) the way the reference evaluates it on a float32 CPU torch
    tensor (processors/migration/velocity_model.py:109-175): constant v0; for
    a gradient, float32 operations in the reference's order.  The final square
    root is torch's CPU float32 sqrt, which is not correctly rounded on every
    input (an ulp off on about 0.7 % of them), so np.sqrt would not reproduce
    the reference's table bit for bit."""
    import torch
    t = np.asarray(t_ms, f32)
    if velocity_type == "constant" or abs(gradient) < 1e-10:
        return np.full(t.shape, v0, f32)
    k = gradient
    tw = t / f32(2000.0)
    z = f32(v0) * tw + f32(0.5 * k * v0) * tw * tw
    z = np.maximum(z, f32(0))
    vs = f32(v0 * v0) + f32(v0 * k) * z + (f32(k * k) * z * z) / f32(3.0)
    v = torch.sqrt(torch.from_numpy(np.maximum(vs, f32(v0 * v0 * 0.5)))).numpy()
    return np.where(t < f32(1.0), f32(v0), v).astype(f32)


def time_domain_rms_torch_port(traces, source_x, source_y, receiver_x, receiver_y, output_x,
                               output_y, n_times, v_rms_in, dt_ms, t_min_ms, max_aperture_m,
                               max_angle_deg, n_il, n_xl, origin_x, origin_y, il_spacing,
                               xl_spacing, azimuth_deg, tile_size=100, sample_batch_size=200,
                               max_traces_per_tile=5000, use_time_dependent_aperture=True,
                               first_tile=0, n_tiles=None):
    """The reference's own float32 torch computation, run on the CPU in the
    reference's order, for a bit-identical result and a faithful CPU timing.

    Steps as kirchhoff_kernel.py:1410-1700 takes them: per tile of consecutive
    output points the midpoint pre-filter and the nearest-``max_traces_per_tile``
    cap (same ``torch.argsort`` call, so ties fall the same way), the input
    samples in batches sized by the reference's memory rule (:1604-1616), the
    per-sample terms of :1243-1282 as whole-tensor float32 operations, and one
    ``scatter_add_`` per batch into the flattened image and fold (the order of
    the float32 sums).  ``first_tile`` / ``n_tiles`` restrict it to a run of
    tiles (a bounded CPU sample).  Returns float32 torch tensors
    (n_times, n_il, n_xl)."""
    import torch
    f = torch.float32
    tr = torch.as_tensor(np.asarray(traces, np.float32))
    sx, sy, rx, ry = (torch.as_tensor(np.asarray(a, np.float32))
                      for a in (source_x, source_y, receiver_x, receiver_y))
    ox = torch.as_tensor(np.asarray(output_x, np.float32))
    oy = torch.as_tensor(np.asarray(output_y, np.float32))
    v = torch.as_tensor(np.asarray(v_rms_in, np.float32))
    n_s = tr.shape[0]
    n_out = n_il * n_xl
    mid_x, mid_y = (sx + rx) / 2.0, (sy + ry) / 2.0
    hoff_sq = ((rx - sx) / 2.0) ** 2 + ((ry - sy) / 2.0) ** 2
    cos_az, sin_az = np.cos(np.radians(azimuth_deg)), np.sin(np.radians(azimuth_deg))
    ddx, ddy = mid_x - origin_x, mid_y - origin_y
    t_il = ((ddx * cos_az + ddy * sin_az) / il_spacing).long().clamp(0, n_il - 1)
    t_xl = ((-ddx * sin_az + ddy * cos_az) / xl_spacing).long().clamp(0, n_xl - 1)
    theta = np.radians(max_angle_deg)
    tan_t = np.tan(theta)
    tile = effective_tile_size(tile_size, max_traces_per_tile, sample_batch_size)
    max_el = int(12.0 * 1024 ** 3 / 4 / 10)
    image = torch.zeros(n_times * n_out, dtype=f)
    fold = torch.zeros(n_times * n_out, dtype=f)
    starts = list(range(0, n_out, tile))[first_tile:]
    if n_tiles is not None:
        starts = starts[:n_tiles]
    with torch.no_grad():
        for a in starts:
            b = min(a + tile, n_out)
            tx, ty = ox[a:b], oy[a:b]
            cx = (tx.min() + tx.max()) / 2
            cy = (ty.min() + ty.max()) / 2
            rad = torch.sqrt(((tx - cx) ** 2 + (ty - cy) ** 2).max())
            dist = torch.sqrt((mid_x - cx) ** 2 + (mid_y - cy) ** 2)
            sel = torch.where(dist < (max_aperture_m + rad + 100))[0]
            if sel.numel() == 0:
                continue
            if sel.numel() > max_traces_per_tile:
                sel = sel[torch.argsort(dist[sel])[:max_traces_per_tile]]
            n_f, n_p = sel.numel(), b - a
            h_sq = (tx[:, None] - mid_x[sel][None, :]) ** 2 + (ty[:, None] - mid_y[sel][None, :]) ** 2
            h = torch.sqrt(h_sq)[None]
            c = (h_sq + hoff_sq[sel][None, :])[None]
            h_sq = h_sq[None]
            cols = (t_il[sel] * n_xl + t_xl[sel]).view(1, 1, n_f)
            sb = min(sample_batch_size, max(10, max_el // max(1, n_p * n_f)), n_s)
            for s0 in range(0, n_s, sb):
                s1 = min(s0 + sb, n_s)
                t_in = 0.0 + torch.arange(s0, s1, dtype=f) * dt_ms
                vb = v[s0:s1]
                v_out = vb.view(-1, 1, 1).expand(s1 - s0, n_p, n_f)
                t_out = torch.sqrt((t_in ** 2).view(-1, 1, 1)
                                   + 4.0 * c * 1e6 / (vb ** 2).view(-1, 1, 1))
                o_idx = (t_out - t_min_ms) / dt_ms
                keep = (o_idx >= 0) & (o_idx < n_times - 0.001)
                if use_time_dependent_aperture:
                    keep = keep & (h < torch.clamp(t_out * v_out / 2000.0 * tan_t,
                                                   max=max_aperture_m))
                else:
                    keep = keep & (h < max_aperture_m)
                z = v_out * t_out / 2000.0
                keep = keep & (torch.atan2(h, z + 1e-6) < theta)
                r2 = z ** 2 + h_sq
                w = z / (torch.sqrt(r2) * r2 + 1e-10)
                amp = tr[s0:s1][:, sel].unsqueeze(1).expand(-1, n_p, -1)
                contrib = amp * w * keep.float()
                lin = o_idx.long().clamp(0, n_times - 1) * n_out + cols
                image.scatter_add_(0, lin.reshape(-1), contrib.reshape(-1))
                fold.scatter_add_(0, lin.reshape(-1), keep.reshape(-1).float())
    return image.view(n_times, n_il, n_xl), fold.view(n_times, n_il, n_xl)
