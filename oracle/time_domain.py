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

The angle mask uses ``np.arctan2`` in float32 where the reference uses torch's;
both are within an ulp or two, so a pair exactly at the angle limit may fall
on either side.  Pinned by golden vectors made by running the reference
(tests/golden/make_time_domain_golden.py).
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
    """V_rms(t) the way the reference evaluates it on a float32 torch tensor
    (processors/migration/velocity_model.py:109-175): constant v0; for a
    gradient, float32 operations in the reference's order."""
    t = np.asarray(t_ms, f32)
    if velocity_type == "constant" or abs(gradient) < 1e-10:
        return np.full(t.shape, v0, f32)
    k = gradient
    tw = t / f32(2000.0)
    z = f32(v0) * tw + f32(0.5 * k * v0) * tw * tw
    z = np.maximum(z, f32(0))
    vs = f32(v0 * v0) + f32(v0 * k) * z + (f32(k * k) * z * z) / f32(3.0)
    v = np.sqrt(np.maximum(vs, f32(v0 * v0 * 0.5)))
    return np.where(t < f32(1.0), f32(v0), v).astype(f32)
