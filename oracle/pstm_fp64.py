"""FP64 CPU oracle for the Kirchhoff PSTM hot path.  TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only as the checker.  The product path
(``seisproc_b200``) never calls it.

This is a float64 numpy restatement of the reference's output-point-centric
Kirchhoff summation, ``migrate_kirchhoff_full``
(processors/migration/kirchhoff_kernel.py:459-854), generalised so that the
velocity may vary with the output point, V = V_rms(t0, x, y):

* depth of the output sample      z = V * t0 / 2               (migration_engine.py:305-306)
* per-leg horizontal distances     h_s = |x - s|, h_r = |x - r|  (kirchhoff_kernel.py:611-626)
* per-leg aperture                 h_s < A and h_r < A           (:635); with the
  time-dependent option A(z) = min(A, z tan(theta))               (:674-680)
* angle mask                       atan2(h, z + 1e-6) < theta, both legs (:670-671, 683-685)
* DSR traveltime                   t = (r_s + r_r) / V, r = sqrt(h^2 + z^2) (:661-662, 688)
* weight (obliquity x spreading)   (z/(r_s+e)) (z/(r_r+e)) / (r_s r_r + e), e = 1e-6 (:690-693)
* sample index                     (t - t_min)/dt clamped to [0, N_s - 1.001] (:707-709)
* linear interpolation             x[i0] + f (x[i0+1] - x[i0])   (:711-721)
* image = sum amp w mask, fold = sum mask                        (:724-730)

The ``clamp='migrator'`` / ``weight='spreading'`` options restate the direct
(non-LUT) branch of ``KirchhoffMigrator._migrate_chunk``
(processors/migration/kirchhoff_migrator.py:362-402): trace time origin 0,
clamp to [0, N_s - 2], weight 1/(sqrt(r_s^2 r_r^2) + 1e-6).

Anti-aliasing (no reference implementation exists; the reference's
``AntialiasFilter`` in processors/migration/antialias.py:48-366 is never
called by a migrator): the triangle filter of half-width L samples evaluated
through the causal double integral of the trace,
    I1[i] = sum_{n<=i} x[n],  I2[i] = sum_{m<i} I1[m],
    y(tau) = (I2~(tau+L) - 2 I2~(tau) + I2~(tau-L)) / L^2,
with I2~ the linear interpolation of I2 (x = 0 outside the trace).  For integer
tau and L this is sum_{|d|<L} (L-|d|) x[tau+d] / L^2; ``triangle_explicit``
restates it by explicit summation.  L = clamp(max(dx |dt/dx|, dy |dt/dy|)/dt_in, 1, L_max)
(Lumley-Claerbout-Bevc operator dip, cited at antialias.py:17-19).
"""
from __future__ import annotations

import numpy as np

EPS = 1e-6

WEIGHTS = ("obliquity_spreading", "spreading", "obliquity", "none")
CLAMPS = ("full", "migrator")


def _as_vgrid(velocity, n_t: int, n_c: int) -> np.ndarray:
    v = np.asarray(velocity, dtype=np.float64)
    if v.ndim == 0:
        return np.full((n_t, n_c), float(v))
    if v.ndim == 1:
        assert v.shape[0] == n_t
        return np.repeat(v[:, None], n_c, 1)
    return v.reshape(n_t, n_c)


def curved_ray_time_s(h, z, v0, k):
    """One-way traveltime (s) in v(z) = v0 + k z along the circular ray,
    arccosh(1 + k r^2 / (2 v0 z)) / k with z floored at 1e-6 m: the reference's
    traveltime table for a velocity gradient (traveltime_lut.py:141-167), which
    the KirchhoffMigrator interpolates bilinearly by default."""
    zs = np.maximum(z, 1e-6)
    arg = np.maximum(1.0 + k * (h * h + zs * zs) / (2.0 * v0 * zs), 1.0)
    return np.arccosh(arg) / k


def _column_terms(xc, yc, sx, sy, rx, ry, z, v, t_out_ms, n_s, in_dt_ms, in_t0_ms, aperture,
                  angle_rad, time_dependent, weight, clamp, ray_gradient=0.0):
    """All per-(trace, t0) quantities for one output column.  Shapes (n_tr, n_t)."""
    hs = np.hypot(xc - sx, yc - sy)[:, None]
    hr = np.hypot(xc - rx, yc - ry)[:, None]
    zz = z[None, :]
    if time_dependent:
        ap = np.minimum(zz * np.tan(angle_rad), aperture)
    else:
        ap = aperture
    if clamp == "migrator":
        zang = np.abs(zz) + EPS
    else:
        zang = zz + EPS
    mask = (hs < ap) & (hr < ap) & (np.arctan2(hs, zang) < angle_rad) & \
           (np.arctan2(hr, zang) < angle_rad)
    rs = np.sqrt(hs * hs + zz * zz)
    rr = np.sqrt(hr * hr + zz * zz)
    if ray_gradient:
        t_ms = 1000.0 * (curved_ray_time_s(hs, zz, v[None, :], ray_gradient) +
                         curved_ray_time_s(hr, zz, v[None, :], ray_gradient))
    else:
        t_ms = (rs + rr) * 1000.0 / v[None, :]
    if clamp == "migrator":
        idx = np.clip(t_ms / in_dt_ms, 0.0, n_s - 2)
    else:
        idx = np.clip((t_ms - in_t0_ms) / in_dt_ms, 0.0, n_s - 1.001)
    if weight == "obliquity_spreading":
        w = (zz / (rs + EPS)) * (zz / (rr + EPS)) / (rs * rr + EPS)
    elif weight == "spreading":
        w = 1.0 / (np.sqrt(rs * rs * rr * rr) + EPS)
    elif weight == "obliquity":
        w = (zz / (rs + EPS)) * (zz / (rr + EPS))
    elif weight == "none":
        w = np.ones_like(rs)
    else:
        raise ValueError(weight)
    return mask, rs, rr, hs, hr, idx, w, t_ms


def _cosine_edge(x, start, end):
    """1 up to ``start``, 0.5 (1 + cos(pi (x - start) / (end - start))) up to
    ``end``, 0 beyond (processors/migration/aperture.py:228-270)."""
    x = np.asarray(x, np.float64)
    out = np.ones_like(x)
    if end > start:
        zone = (x > start) & (x <= end)
        out = np.where(zone, 0.5 * (1.0 + np.cos(np.pi * (x - start) / (end - start))), out)
    return np.where(x > end, 0.0, out)


def distance_taper_fp64(h, max_distance, taper_width):
    """ApertureController._compute_distance_taper (aperture.py:228-249)."""
    return _cosine_edge(h, max_distance * (1.0 - taper_width), max_distance)


def angle_taper_fp64(angle_rad, max_angle_rad, taper_width):
    """ApertureController._compute_angle_taper (aperture.py:251-270)."""
    return _cosine_edge(angle_rad, max_angle_rad * (1.0 - taper_width), max_angle_rad)


def offset_taper_fp64(offset, min_offset, max_offset, taper_width):
    """ApertureController._compute_offset_mask (aperture.py:197-226): 0 outside
    [min, max], cosine rise over the first taper_width of the range and fall
    over the last."""
    o = np.asarray(offset, np.float64)
    rng = taper_width * (max_offset - min_offset)
    near = np.ones_like(o)
    far = np.ones_like(o)
    if rng > 0:
        zn = (o >= min_offset) & (o < min_offset + rng)
        near = np.where(zn, 0.5 * (1.0 - np.cos(np.pi * (o - min_offset) / rng)), 1.0)
        zf = (o > max_offset - rng) & (o <= max_offset)
        far = np.where(zf, 0.5 * (1.0 + np.cos(np.pi * (o - (max_offset - rng)) / rng)), 1.0)
    return np.where((o >= min_offset) & (o <= max_offset), near * far, 0.0)


def aperture_taper_fp64(hs, hr, z, aperture, angle_rad, taper_width):
    """Distance and angle tapers of both legs, angle = atan2(h, |z|)
    (ApertureController.compute_aperture_mask, aperture.py:65-147, without its
    offset factor).  hs, hr: (n_tr, 1); z: (1, n_t)."""
    az = np.abs(z)
    return (distance_taper_fp64(hs, aperture, taper_width) *
            distance_taper_fp64(hr, aperture, taper_width) *
            angle_taper_fp64(np.arctan2(hs, az), angle_rad, taper_width) *
            angle_taper_fp64(np.arctan2(hr, az), angle_rad, taper_width))


def _candidates(xc, yc, sx, sy, rx, ry, aperture):
    """Traces whose legs are both inside the (largest) aperture of a column."""
    hs = np.hypot(xc - sx, yc - sy)
    hr = np.hypot(xc - rx, yc - ry)
    return np.nonzero((hs < aperture) & (hr < aperture))[0]


def _aa_halfwidth(xc, yc, sx, sy, rx, ry, rs, rr, v, dx_out, dy_out, in_dt_ms, l_max):
    """Triangle half-width in input samples from the operator dip (both output axes)."""
    qs = 1.0 / rs
    qr = 1.0 / rr
    gx = ((xc - sx)[:, None] * qs + (xc - rx)[:, None] * qr) / v[None, :]
    gy = ((yc - sy)[:, None] * qs + (yc - ry)[:, None] * qr) / v[None, :]
    lx = np.abs(gx) * dx_out
    ly = np.abs(gy) * dy_out
    return np.clip(np.maximum(lx, ly) * 1000.0 / in_dt_ms, 1.0, l_max)


def double_integral(tr: np.ndarray) -> np.ndarray:
    """I2[i] = sum_{m<i} I1[m] for i = 0..N (row per trace), I1 = inclusive cumsum."""
    i1 = np.cumsum(tr, axis=-1)
    i2 = np.zeros(tr.shape[:-1] + (tr.shape[-1] + 1,))
    i2[..., 1:] = np.cumsum(i1, axis=-1)
    return i2


def _i2_interp(i2: np.ndarray, i1_last: float, pos: np.ndarray) -> np.ndarray:
    """Linear interpolation of the extended I2 sequence (0 below 0, linear past N)."""
    n = i2.shape[0] - 1
    p0 = np.floor(pos)
    f = pos - p0
    p0 = p0.astype(np.int64)

    def at(k):
        k = np.asarray(k)
        out = np.where(k <= 0, 0.0, 0.0)
        inside = (k > 0) & (k <= n)
        out = np.where(inside, i2[np.clip(k, 0, n)], out)
        out = np.where(k > n, i2[n] + (k - n) * i1_last, out)
        return out

    return at(p0) * (1.0 - f) + at(p0 + 1) * f


def triangle_explicit(tr: np.ndarray, i: int, L: int) -> float:
    """Explicit-sum triangle filter: sum_{|d|<L} (L-|d|) x[i+d] / L^2 (x = 0 outside)."""
    s = 0.0
    for d in range(-L + 1, L):
        j = i + d
        if 0 <= j < tr.shape[0]:
            s += (L - abs(d)) * tr[j]
    return s / (L * L)


def migrate_fp64(traces, sx, sy, rx, ry, out_x, out_y, t_out_ms, velocity, in_dt_ms,
                 in_t0_ms, aperture, angle_deg, time_dependent=False,
                 weight="obliquity_spreading", clamp="full", antialias=False, dx_out=0.0,
                 dy_out=0.0, l_max=32.0, columns=None, taper_width=0.0, ray_gradient=0.0):
    """Forward migration (data -> image) in float64.

    traces: (N_s, N_tr); coordinates float64 (any common origin);
    out_x/out_y: (n_c,) column coordinates; t_out_ms: (N_t,) output times;
    velocity: scalar, (N_t,) or (N_t, n_c) V_rms at the output samples.
    Returns image (N_t, n_c) and fold (N_t, n_c) as float64.
    ``columns`` optionally restricts the computation to a subset of columns
    (others stay 0).  ``taper_width`` > 0 multiplies every weight by the
    aperture controller's distance and angle cosine tapers of both legs
    (``aperture_taper_fp64``); the fold still counts the hard-masked pairs.
    ``ray_gradient`` k != 0 replaces the straight-ray traveltime by the curved
    ray of v(z) = v0 + k z (``curved_ray_time_s``), v0 = ``velocity`` (constant).
    """
    tr = np.asarray(traces, dtype=np.float64)
    n_s, n_tr = tr.shape
    out_x = np.asarray(out_x, np.float64)
    out_y = np.asarray(out_y, np.float64)
    t_out_ms = np.asarray(t_out_ms, np.float64)
    n_t, n_c = t_out_ms.shape[0], out_x.shape[0]
    vg = _as_vgrid(velocity, n_t, n_c)
    sx, sy, rx, ry = (np.asarray(a, np.float64) for a in (sx, sy, rx, ry))
    ang = np.radians(angle_deg)
    image = np.zeros((n_t, n_c))
    fold = np.zeros((n_t, n_c))
    if n_tr == 0:
        return image, fold
    trT = tr.T  # (n_tr, n_s)
    if antialias:
        i2 = double_integral(trT)
        i1_last = np.cumsum(trT, axis=-1)[:, -1]
    cols = range(n_c) if columns is None else columns
    rows = np.arange(n_tr)[:, None]
    for c in cols:
        v = vg[:, c]
        z = v * (t_out_ms / 1000.0) / 2.0
        cand = _candidates(out_x[c], out_y[c], sx, sy, rx, ry, aperture)
        if cand.size == 0:
            continue
        mask, rs, rr, hs, hr, idx, w, _ = _column_terms(
            out_x[c], out_y[c], sx[cand], sy[cand], rx[cand], ry[cand], z, v, t_out_ms, n_s,
            in_dt_ms, in_t0_ms, aperture, ang, time_dependent, weight, clamp, ray_gradient)
        if taper_width > 0:
            w = w * aperture_taper_fp64(hs, hr, z[None, :], aperture, ang, taper_width)
        keep = np.nonzero(mask.any(axis=1))[0]
        if keep.size == 0:
            continue
        sel = cand[keep]
        m = mask[keep]
        rs, rr, idx, w = rs[keep], rr[keep], idx[keep], w[keep]
        if antialias:
            L = _aa_halfwidth(out_x[c], out_y[c], sx[sel], sy[sel], rx[sel], ry[sel], rs, rr, v,
                              dx_out, dy_out, in_dt_ms, l_max)
            amp = np.empty_like(idx)
            for q, j in enumerate(sel):
                y0 = _i2_interp(i2[j], i1_last[j], idx[q] + L[q])
                y1 = _i2_interp(i2[j], i1_last[j], idx[q])
                y2 = _i2_interp(i2[j], i1_last[j], idx[q] - L[q])
                amp[q] = (y0 - 2.0 * y1 + y2) / (L[q] * L[q])
        else:
            ix = idx
            i0 = np.floor(ix).astype(np.int64)
            i1 = np.minimum(i0 + 1, n_s - 1)
            f = ix - i0
            a0 = trT[sel[:, None], i0]
            a1 = trT[sel[:, None], i1]
            amp = a0 + f * (a1 - a0)
        image[:, c] = np.sum(np.where(m, amp * w, 0.0), axis=0)
        fold[:, c] = np.sum(m, axis=0)
    return image, fold


def demigrate_fp64(image, n_s, sx, sy, rx, ry, out_x, out_y, t_out_ms, velocity, in_dt_ms,
                   in_t0_ms, aperture, angle_deg, time_dependent=False,
                   weight="obliquity_spreading", clamp="full"):
    """Adjoint of ``migrate_fp64`` (image -> data): the transpose of the linear
    interpolation scatters w * m into samples i0 and i0+1.  Returns (N_s, N_tr)."""
    image = np.asarray(image, np.float64)
    out_x = np.asarray(out_x, np.float64)
    out_y = np.asarray(out_y, np.float64)
    t_out_ms = np.asarray(t_out_ms, np.float64)
    n_t, n_c = t_out_ms.shape[0], out_x.shape[0]
    vg = _as_vgrid(velocity, n_t, n_c)
    sx, sy, rx, ry = (np.asarray(a, np.float64) for a in (sx, sy, rx, ry))
    n_tr = sx.shape[0]
    ang = np.radians(angle_deg)
    data = np.zeros((n_tr, n_s))
    flat = data.reshape(-1)
    for c in range(n_c):
        v = vg[:, c]
        z = v * (t_out_ms / 1000.0) / 2.0
        mask, rs, rr, hs, hr, idx, w, _ = _column_terms(
            out_x[c], out_y[c], sx, sy, rx, ry, z, v, t_out_ms, n_s, in_dt_ms, in_t0_ms,
            aperture, ang, time_dependent, weight, clamp)
        g = np.where(mask, w * image[None, :, c], 0.0)
        i0 = np.floor(idx).astype(np.int64)
        i1 = np.minimum(i0 + 1, n_s - 1)
        f = idx - i0
        base = (np.arange(n_tr) * n_s)[:, None]
        np.add.at(flat, (base + i0).ravel(), (g * (1.0 - f)).ravel())
        np.add.at(flat, (base + i1).ravel(), (g * f).ravel())
    return data.T.copy()


def vgrad_fp64(traces, grad_image, sx, sy, rx, ry, out_x, out_y, t_out_ms, velocity, in_dt_ms,
               in_t0_ms, aperture, angle_deg, time_dependent=False):
    """d<grad_image, migrate(traces; V)>/dV(t0, x, y) for the obliquity x spreading
    operator, differentiating traveltime and weight (masks held fixed; the clamped
    tail of the trace has zero time derivative).  Weight taken as z^2/(r_s^2 r_r^2)."""
    tr = np.asarray(traces, np.float64)
    n_s, n_tr = tr.shape
    out_x = np.asarray(out_x, np.float64)
    out_y = np.asarray(out_y, np.float64)
    t_out_ms = np.asarray(t_out_ms, np.float64)
    n_t, n_c = t_out_ms.shape[0], out_x.shape[0]
    vg = _as_vgrid(velocity, n_t, n_c)
    sx, sy, rx, ry = (np.asarray(a, np.float64) for a in (sx, sy, rx, ry))
    ang = np.radians(angle_deg)
    gv = np.zeros((n_t, n_c))
    trT = tr.T
    hi = n_s - 1.001
    for c in range(n_c):
        v = vg[:, c]
        z = v * (t_out_ms / 1000.0) / 2.0
        mask, rs, rr, hs, hr, idx, w, t_ms = _column_terms(
            out_x[c], out_y[c], sx, sy, rx, ry, z, v, t_out_ms, n_s, in_dt_ms, in_t0_ms,
            aperture, ang, time_dependent, "obliquity_spreading", "full")
        raw = (t_ms - in_t0_ms) / in_dt_ms
        i0 = np.floor(idx).astype(np.int64)
        f = idx - i0
        a0 = trT[np.arange(n_tr)[:, None], i0]
        a1 = trT[np.arange(n_tr)[:, None], np.minimum(i0 + 1, n_s - 1)]
        amp = a0 + f * (a1 - a0)
        slope = np.where((raw > 0.0) & (raw < hi), a1 - a0, 0.0)
        zz = z[None, :]
        vv = v[None, :]
        w0 = zz * zz / (rs * rs * rr * rr)
        dw = 2.0 * w0 / vv * (1.0 - zz * zz * (1.0 / (rs * rs) + 1.0 / (rr * rr)))
        dt_dv = -(hs * hs / rs + hr * hr / rr) / (vv * vv)  # seconds per (m/s)
        didx = dt_dv * 1000.0 / in_dt_ms
        contrib = np.where(mask, amp * dw + w0 * slope * didx, 0.0)
        gv[:, c] = np.asarray(grad_image)[:, c] * contrib.sum(axis=0)
    return gv


def count_pairs_fp64(sx, sy, rx, ry, out_x, out_y, t_out_ms, velocity, aperture, angle_deg,
                     time_dependent=False):
    """Exact number of contributing (output sample, trace) pairs (mask count)."""
    out_x = np.asarray(out_x, np.float64)
    out_y = np.asarray(out_y, np.float64)
    sx, sy, rx, ry = (np.asarray(a, np.float64) for a in (sx, sy, rx, ry))
    t_out_ms = np.asarray(t_out_ms, np.float64)
    n_t, n_c = t_out_ms.shape[0], out_x.shape[0]
    vg = _as_vgrid(velocity, n_t, n_c)
    ang = np.radians(angle_deg)
    total = 0
    for c in range(n_c):
        v = vg[:, c]
        z = v * (t_out_ms / 1000.0) / 2.0
        cand = _candidates(out_x[c], out_y[c], sx, sy, rx, ry, aperture)
        hs = np.hypot(out_x[c] - sx[cand], out_y[c] - sy[cand])[:, None]
        hr = np.hypot(out_x[c] - rx[cand], out_y[c] - ry[cand])[:, None]
        ap = np.minimum(z * np.tan(ang), aperture)[None, :] if time_dependent else aperture
        m = (hs < ap) & (hr < ap) & (np.arctan2(hs, z[None, :] + EPS) < ang) & \
            (np.arctan2(hr, z[None, :] + EPS) < ang)
        total += int(m.sum())
    return total


def normalize_by_fold_fp64(image, fold, min_fold=1):
    """image/fold where fold >= min_fold, else unchanged (kirchhoff_kernel.py:437-456)."""
    out = np.array(image, dtype=np.float64, copy=True)
    m = fold >= min_fold
    out[m] = out[m] / fold[m]
    return out
