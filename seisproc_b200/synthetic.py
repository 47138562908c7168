"""Seeded synthetic surveys for the Kirchhoff PSTM workloads.

Every generator is deterministic for a given seed.  Geometry and diffractor
parameters come from ``numpy.random.RandomState`` (float64), trace samples are
synthesised with torch on the requested device, and the additive noise comes
from a counter-based integer hash, so the same (seed, trace, sample) triple
always yields the same noise value on the CPU and on the GPU (up to the last
ulp of ``log``/``cos``).

Workloads (sizes follow the reference PSTM configurations; none of them is a
public dataset):

* ``survey_2d``: 12 common-offset sections (offsets 0..1100 m step 100), 240
  CMPs at 12.5 m, 501 samples at 4 ms, 40 diffractors, V = 2000 m/s, Ricker
  25 Hz, 5 % RMS noise.
* ``survey_3d``: N traces with midpoints uniform on a square, offsets uniform,
  azimuths uniform, 1000 samples at 4 ms, 200 diffractors, Ricker 30 Hz, 3 %
  RMS noise, V_rms(t0, x, y) rising 1500 -> 3500 m/s with a +-5 % lateral
  sinusoid.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional, Tuple

import math
import numpy as np
import torch

_MASK32 = 0xFFFFFFFF


def _mix32(x: torch.Tensor) -> torch.Tensor:
    """32-bit avalanche mix (Wellons' "lowbias32" xorshift-multiply family).

    Operates on int64 tensors holding values in [0, 2**32); every product stays
    below 2**63 so the arithmetic is exact on every torch device.
    """
    x = x & _MASK32
    x = x ^ (x >> 16)
    x = (x * 0x7FEB352D) & _MASK32
    x = x ^ (x >> 15)
    x = (x * 0x846CA68B) & _MASK32
    x = x ^ (x >> 16)
    return x


def hashed_gaussian(seed: int, trace_ids: torch.Tensor, n_samples: int) -> torch.Tensor:
    """Standard-normal noise of shape (n_samples, n_traces), keyed by (seed, trace, sample).

    Box-Muller on two hashed uniforms.  ``trace_ids`` is an int64 tensor; the
    result lives on its device.
    """
    dev = trace_ids.device
    s = torch.arange(n_samples, device=dev, dtype=torch.int64).view(-1, 1)
    j = trace_ids.view(1, -1).to(torch.int64)
    key = _mix32(j * 0x9E3779B1 + (seed & _MASK32))
    key = _mix32(key ^ (s * 0x85EBCA77 & _MASK32))
    u1 = (_mix32(key ^ 0x68E31DA4).to(torch.float64) + 1.0) / 4294967297.0
    u2 = _mix32(key ^ 0xB5297A4D).to(torch.float64) / 4294967296.0
    g = torch.sqrt(-2.0 * torch.log(u1)) * torch.cos(2.0 * math.pi * u2)
    return g.to(torch.float32)


def ricker(tau: torch.Tensor, f_peak: float) -> torch.Tensor:
    a = (math.pi * f_peak * tau) ** 2
    return (1.0 - 2.0 * a) * torch.exp(-a)


@dataclass
class Survey:
    """A synthetic pre-stack dataset in the reference's conventions.

    ``traces`` is (n_samples, n_traces) float32 (sample-major, as the reference
    migration API takes it).  Coordinates are float64 world coordinates.
    """
    traces: torch.Tensor
    source_x: np.ndarray
    source_y: np.ndarray
    receiver_x: np.ndarray
    receiver_y: np.ndarray
    dt_ms: float
    t_min_ms: float
    # output grid
    origin_x: float
    origin_y: float
    il_spacing: float
    xl_spacing: float
    n_il: int
    n_xl: int
    n_times: int
    max_aperture_m: float
    max_angle_deg: float
    # velocity: either a constant or a (n_times, n_il, n_xl) V_rms cube at output points
    velocity_mps: float = 2000.0
    vrms: Optional[np.ndarray] = None
    diffractors: dict = field(default_factory=dict)

    @property
    def n_traces(self) -> int:
        return int(self.traces.shape[1])

    @property
    def n_samples(self) -> int:
        return int(self.traces.shape[0])


def _synthesise(src: np.ndarray, rcv: np.ndarray, dif_xy: np.ndarray, dif_t0: np.ndarray,
                dif_v: np.ndarray, dif_amp: np.ndarray, n_samples: int, dt_ms: float,
                f_peak: float, noise_rel: float, seed: int, device,
                chunk: int = 8192) -> torch.Tensor:
    """Sum of Ricker diffraction responses at DSR times, plus hashed noise.

    Each (trace, diffractor) pair contributes a windowed wavelet (+-3/f around
    its arrival); windows are scatter-added so the cost is O(traces x diffractors
    x window), not O(traces x diffractors x samples).
    """
    dev = torch.device(device)
    n_tr = src.shape[0]
    out = torch.zeros(n_tr, n_samples, dtype=torch.float32, device=dev)
    dt = dt_ms * 1e-3
    half = int(math.ceil(1.5 / f_peak / dt)) + 1
    win = torch.arange(-half, half + 1, device=dev, dtype=torch.float64)
    dxy = torch.from_numpy(dif_xy).to(dev)
    t0 = torch.from_numpy(dif_t0).to(dev)
    v = torch.from_numpy(dif_v).to(dev)
    amp = torch.from_numpy(dif_amp).to(dev)
    tau2 = (0.5 * t0) ** 2
    for a in range(0, n_tr, chunk):
        b = min(n_tr, a + chunk)
        s = torch.from_numpy(src[a:b]).to(dev)
        r = torch.from_numpy(rcv[a:b]).to(dev)
        hs2 = ((s[:, None, :] - dxy[None, :, :]) ** 2).sum(-1)
        hr2 = ((r[:, None, :] - dxy[None, :, :]) ** 2).sum(-1)
        t = torch.sqrt(tau2 + hs2 / v ** 2) + torch.sqrt(tau2 + hr2 / v ** 2)  # (nb, nd) seconds
        c = torch.floor(t / dt)
        idx = c[..., None] + win  # (nb, nd, W)
        val = amp[None, :, None] * ricker(idx * dt - t[..., None], f_peak)
        ok = (idx >= 0) & (idx < n_samples)
        rows = torch.arange(a, b, device=dev).view(-1, 1, 1).expand_as(idx)
        flat = (rows - a) * n_samples + idx.clamp(0, n_samples - 1).long()
        blk = torch.zeros((b - a) * n_samples, dtype=torch.float64, device=dev)
        blk.index_put_((flat[ok],), val[ok], accumulate=True)
        out[a:b] = blk.view(b - a, n_samples).to(torch.float32)
    traces = out.t().contiguous()  # (n_samples, n_tr)
    if noise_rel > 0:
        rms = float(torch.sqrt((traces.double() ** 2).mean()).item())
        ids = torch.arange(n_tr, device=dev, dtype=torch.int64)
        for a in range(0, n_tr, 65536):
            b = min(n_tr, a + 65536)
            traces[:, a:b] += (noise_rel * rms) * hashed_gaussian(seed, ids[a:b], n_samples)
    return traces


def survey_2d(seed: int = 1234, device="cpu", n_offsets: int = 12, n_cmp: int = 240,
              n_samples: int = 501, n_diffractors: int = 40) -> Survey:
    """2D common-offset sections over point diffractors, constant V = 2000 m/s."""
    rs = np.random.RandomState(seed)
    dx = 12.5
    x = np.arange(n_cmp) * dx
    offs = np.arange(n_offsets) * 100.0
    mx = np.tile(x, n_offsets)
    h = np.repeat(offs, n_cmp)
    src = np.stack([mx - h / 2, np.zeros_like(mx)], 1)
    rcv = np.stack([mx + h / 2, np.zeros_like(mx)], 1)
    v = 2000.0
    dxs = rs.uniform(0.0, x[-1], n_diffractors)
    dt0 = rs.uniform(0.3, 1.8, n_diffractors)
    damp = rs.uniform(0.5, 1.5, n_diffractors) * np.where(rs.rand(n_diffractors) < 0.5, -1.0, 1.0)
    dif_xy = np.stack([dxs, np.zeros_like(dxs)], 1)
    traces = _synthesise(src, rcv, dif_xy, dt0, np.full(n_diffractors, v), damp, n_samples, 4.0,
                         25.0, 0.05, seed, device)
    return Survey(traces=traces, source_x=src[:, 0], source_y=src[:, 1], receiver_x=rcv[:, 0],
                  receiver_y=rcv[:, 1], dt_ms=4.0, t_min_ms=0.0, origin_x=0.0, origin_y=0.0,
                  il_spacing=dx, xl_spacing=dx, n_il=n_cmp, n_xl=1, n_times=n_samples,
                  max_aperture_m=1500.0, max_angle_deg=60.0, velocity_mps=v,
                  diffractors=dict(x=dxs, t0=dt0, amp=damp))


def vrms_3d(t0_s: np.ndarray, x: np.ndarray, y: np.ndarray, t_max_s: float,
            extent: float = 5000.0) -> np.ndarray:
    """V_rms(t0, x, y) = (1500 + 2000 t0/t_max) (1 + 0.05 sin(2 pi x/L) sin(2 pi y/L));
    a single output time (t_max = 0) takes the 1500 m/s trend value."""
    ramp = 2000.0 * t0_s / t_max_s if t_max_s > 0 else 0.0 * t0_s
    return (1500.0 + ramp) * (
        1.0 + 0.05 * np.sin(2 * np.pi * x / extent) * np.sin(2 * np.pi * y / extent))


def survey_3d(n_traces: int = 500_000, seed: int = 2025, device="cpu", n_samples: int = 1000,
              dt_ms: float = 4.0, extent: float = 5000.0, max_offset: float = 3000.0,
              n_il: int = 200, n_xl: int = 200, spacing: float = 25.0,
              n_diffractors: int = 200, aperture: float = 1000.0, angle: float = 60.0,
              noise_rel: float = 0.03, f_peak: float = 30.0, n_times: Optional[int] = None,
              utm_origin: Tuple[float, float] = (0.0, 0.0), lateral_velocity: bool = True,
              midpoint_box: Optional[Tuple[float, float, float, float]] = None,
              offset_range: Optional[Tuple[float, float]] = None,
              azimuth_range: Optional[Tuple[float, float]] = None,
              diffractor_seed: Optional[int] = None) -> Survey:
    """3D survey: uniform midpoints/offsets/azimuths over point diffractors.

    ``utm_origin`` is added to every world coordinate (float64) to exercise
    tile-local coordinate handling; the output grid origin moves with it.
    ``midpoint_box`` (x0, x1, y0, y1) restricts midpoints (used for crops);
    ``offset_range`` (m) and ``azimuth_range`` (radians) restrict the offsets
    and azimuths (used to draw one offset/azimuth class).
    """
    rs = np.random.RandomState(seed)
    if midpoint_box is None:
        midpoint_box = (0.0, extent, 0.0, extent)
    mx = rs.uniform(midpoint_box[0], midpoint_box[1], n_traces)
    my = rs.uniform(midpoint_box[2], midpoint_box[3], n_traces)
    o0, o1 = offset_range if offset_range is not None else (0.0, max_offset)
    a0, a1 = azimuth_range if azimuth_range is not None else (0.0, 2 * np.pi)
    off = rs.uniform(o0, o1, n_traces)
    az = rs.uniform(a0, a1, n_traces)
    hx, hy = 0.5 * off * np.cos(az), 0.5 * off * np.sin(az)
    src = np.stack([mx - hx, my - hy], 1)
    rcv = np.stack([mx + hx, my + hy], 1)
    nt = n_samples if n_times is None else n_times
    t_max = (nt - 1) * dt_ms * 1e-3
    drs = np.random.RandomState(seed + 1 if diffractor_seed is None else diffractor_seed)
    dxy = np.stack([drs.uniform(0, extent, n_diffractors), drs.uniform(0, extent, n_diffractors)], 1)
    dt0 = drs.uniform(0.2, 0.9 * t_max, n_diffractors)
    damp = drs.uniform(0.5, 1.5, n_diffractors) * np.where(drs.rand(n_diffractors) < 0.5, -1.0, 1.0)
    if lateral_velocity:
        dv = vrms_3d(dt0, dxy[:, 0], dxy[:, 1], t_max, extent)
    else:
        dv = 1500.0 + 2000.0 * dt0 / t_max
    traces = _synthesise(src, rcv, dxy, dt0, dv, damp, n_samples, dt_ms, f_peak, noise_rel, seed,
                         device)
    ox, oy = utm_origin
    # output grid: n_il x n_xl at `spacing`, centred on the survey square
    gx0 = 0.5 * (extent - (n_il - 1) * spacing)
    gy0 = 0.5 * (extent - (n_xl - 1) * spacing)
    t0 = np.arange(nt) * dt_ms * 1e-3
    if lateral_velocity:
        cx = gx0 + np.arange(n_il) * spacing
        cy = gy0 + np.arange(n_xl) * spacing
        vr = vrms_3d(t0[:, None, None], cx[None, :, None], cy[None, None, :], t_max, extent)
    else:
        vr = np.broadcast_to((1500.0 + 2000.0 * t0 / t_max)[:, None, None], (nt, n_il, n_xl))
    return Survey(traces=traces, source_x=src[:, 0] + ox, source_y=src[:, 1] + oy,
                  receiver_x=rcv[:, 0] + ox, receiver_y=rcv[:, 1] + oy, dt_ms=dt_ms, t_min_ms=0.0,
                  origin_x=gx0 + ox, origin_y=gy0 + oy, il_spacing=spacing, xl_spacing=spacing,
                  n_il=n_il, n_xl=n_xl, n_times=nt, max_aperture_m=aperture, max_angle_deg=angle,
                  velocity_mps=float(vr.mean()), vrms=np.ascontiguousarray(vr, dtype=np.float32),
                  diffractors=dict(xy=dxy, t0=dt0, amp=damp, v=dv))


def survey_classes(counts, seed: int = 64, n_offset_bins: int = 8, n_azimuth_bins: int = 8,
                   max_offset: float = 3000.0, device="cpu", **kw):
    """Offset/azimuth classes (offset-major) of one synthetic survey, class i
    holding counts[i] traces drawn from its own offset bin and azimuth sector;
    all classes share the diffractors, velocity and output grid."""
    out = []
    for i, n in enumerate(counts):
        ob, ab = divmod(i, n_azimuth_bins)
        out.append(survey_3d(
            n_traces=int(n), seed=seed * 1000 + i, device=device, max_offset=max_offset,
            offset_range=(ob * max_offset / n_offset_bins, (ob + 1) * max_offset / n_offset_bins),
            azimuth_range=(ab * 2 * np.pi / n_azimuth_bins, (ab + 1) * 2 * np.pi / n_azimuth_bins),
            diffractor_seed=seed + 1, **kw))
    return out


def class_counts_loguniform(n_classes: int = 64, lo: int = 2000, hi: int = 40000,
                            seed: int = 64) -> np.ndarray:
    """Trace counts per offset/azimuth class, log-uniform in [lo, hi]."""
    rs = np.random.RandomState(seed)
    return np.exp(rs.uniform(np.log(lo), np.log(hi), n_classes)).astype(np.int64)
