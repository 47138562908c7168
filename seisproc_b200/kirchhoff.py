"""Torch-facing PSTM operators over libseispstm (CUDA sm_100a).

* ``PSTMPlan``: one survey geometry + output grid + migration parameters on the
  device; owns the plan's scratch (sorted geometry, per-tile trace lists, staged
  traces).  Its methods launch the kernels on the current torch CUDA stream.
* ``migrate_kirchhoff_full``: the reference's output-point-centric Kirchhoff
  summation signature (processors/migration/kirchhoff_kernel.py:459-504), torch
  tensors in and out, plus an optional V_rms tensor for ``velocity``.
* ``normalize_by_fold``: image / fold where fold >= min_fold
  (kirchhoff_kernel.py:437-456).

No CPU fallback exists: every entry point requires a CUDA device and the
compiled library.
"""
from __future__ import annotations

import ctypes as C
import logging
import math
import time
from typing import Callable, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from .kernel_backend import require_cuda

logger = logging.getLogger(__name__)

WEIGHTS = {"obliquity_spreading": _lib.WEIGHT_OBLIQUITY_SPREADING,
           "spreading": _lib.WEIGHT_SPREADING, "obliquity": _lib.WEIGHT_OBLIQUITY,
           "none": _lib.WEIGHT_NONE}
CLAMPS = {"full": _lib.CLAMP_FULL, "migrator": _lib.CLAMP_MIGRATOR}
STORAGES = {"f32": _lib.PSTM_F32, "float32": _lib.PSTM_F32, "bf16": _lib.PSTM_BF16,
            "bfloat16": _lib.PSTM_BF16, "f16": _lib.PSTM_F16, "float16": _lib.PSTM_F16}


def _stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def velocity_strides(v: torch.Tensor, n_times: int, n_cols: int) -> Tuple[torch.Tensor, int, int]:
    """Device velocity tensor and its (stride over output samples, stride over
    columns): constant, V(t0) or V(t0, column)."""
    v = v.to(torch.float32).contiguous()
    if v.numel() == 1:
        return v.reshape(1), 0, 0
    if v.dim() == 1:
        if v.shape[0] != n_times:
            raise ValueError(f"1D velocity must have n_times={n_times} samples, got {v.shape[0]}")
        return v, 1, 0
    flat = v.reshape(v.shape[0], -1)
    if flat.shape != (n_times, n_cols):
        raise ValueError(f"velocity must be (n_times, n_il, n_xl) = ({n_times}, {n_cols} columns),"
                         f" got {tuple(v.shape)}")
    return flat, n_cols, 1


class PSTMPlan:
    """A migration plan on the current CUDA device.

    Coordinates may be float32 or float64 (world, e.g. UTM); the grid origin is
    subtracted in float64 on the device and everything downstream is grid-local
    float32.  ``forward_only=True`` is for plans that only migrate: float32
    traces are staged in intercept form (one FMA per interpolation tap, ~3 %
    faster); ``demigrate`` then matches the migration's transpose to ~1e-5
    rather than to float rounding, and ``velocity_gradient`` refuses the plan
    (a batch takes it when all of its class plans are forward_only).  ``taper_width`` in (0, 1) adds the aperture controller's
    distance and angle cosine tapers of both legs (migration only, float32).
    ``ray_gradient`` k != 0 takes curved-ray traveltimes in v(z) = v0 + k z
    (the velocity passed is v0), as the reference migrator's default table.
    """

    def __init__(self, source_x, source_y, receiver_x, receiver_y, *, n_il: int, n_xl: int,
                 n_times: int, origin_x: float, origin_y: float, il_dx: float, il_dy: float,
                 xl_dx: float, xl_dy: float, t0_ms: float, dt_ms: float, n_samples: int,
                 in_t0_ms: float, in_dt_ms: float, max_aperture_m: float, max_angle_deg: float,
                 time_dependent_aperture: bool = False, weight: str = "obliquity_spreading",
                 clamp: str = "full", storage: str = "f32", variant: int = 0,
                 kernel_backend=None, antialias: bool = False, aa_dx: float = 0.0,
                 aa_dy: float = 0.0, aa_max_halfwidth: float = 32.0,
                 forward_only: bool = False, taper_width: float = 0.0,
                 ray_gradient: float = 0.0):
        require_cuda(kernel_backend)
        self._lib = _lib.lib()
        self._handle = C.c_void_p(None)
        dev = torch.device("cuda", torch.cuda.current_device())
        coords = []
        for a in (source_x, source_y, receiver_x, receiver_y):
            t = torch.as_tensor(a)
            if t.dtype not in (torch.float32, torch.float64):
                t = t.to(torch.float64)
            coords.append(t.to(dev).contiguous())
        dt = coords[0].dtype
        coords = [c.to(dt) for c in coords]
        n_tr = coords[0].numel()
        if any(c.numel() != n_tr for c in coords):
            raise ValueError("source/receiver coordinate arrays must have the same length")
        if weight not in WEIGHTS:
            raise ValueError(f"unknown weight {weight!r}")
        if clamp not in CLAMPS:
            raise ValueError(f"unknown clamp {clamp!r}")
        if storage not in STORAGES:
            raise ValueError(f"unknown storage {storage!r}")
        self.grid = _lib.Grid(n_il, n_xl, n_times, origin_x, origin_y, il_dx, il_dy, xl_dx, xl_dy,
                              t0_ms, dt_ms)
        self.params = _lib.Params(n_samples, in_t0_ms, in_dt_ms, max_aperture_m, max_angle_deg,
                                  int(bool(time_dependent_aperture)), WEIGHTS[weight],
                                  CLAMPS[clamp], STORAGES[storage], int(bool(antialias)),
                                  float(aa_dx), float(aa_dy), float(aa_max_halfwidth),
                                  int(variant), int(bool(forward_only)), float(taper_width),
                                  float(ray_gradient))
        geo = _lib.Geometry(n_tr, _lib.PSTM_F64 if dt == torch.float64 else _lib.PSTM_F32,
                            *[c.data_ptr() for c in coords])
        _lib.check(self._lib.pstm_plan_create(C.byref(self._handle), C.byref(self.grid),
                                              C.byref(self.params), C.byref(geo),
                                              _stream_handle()))
        self.n_il, self.n_xl, self.n_times = n_il, n_xl, n_times
        self.n_cols = n_il * n_xl
        self.n_samples = n_samples
        self.n_traces = n_tr
        self.device = dev
        self.weight = weight
        self.storage = storage

    # ------------------------------------------------------------ plumbing --
    def close(self):
        if getattr(self, "_handle", None) is not None and self._handle.value:
            self._lib.pstm_plan_destroy(self._handle)
            self._handle = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self) -> dict:
        s = _lib.PlanStats()
        _lib.check(self._lib.pstm_plan_get_stats(self._handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def check(self) -> None:
        """Synchronise and raise if a device-side check fired."""
        _lib.check(self._lib.pstm_check(self._handle, _stream_handle()))

    def _vel(self, velocity) -> Tuple[torch.Tensor, int, int]:
        if not torch.is_tensor(velocity):
            velocity = torch.as_tensor(np.asarray(velocity, np.float32))
        return velocity_strides(velocity.to(self.device), self.n_times, self.n_cols)

    def _traces(self, traces: torch.Tensor, trace_major: bool) -> torch.Tensor:
        t = traces.to(self.device, torch.float32).contiguous()
        want = (self.n_traces, self.n_samples) if trace_major else (self.n_samples, self.n_traces)
        if tuple(t.shape) != want:
            raise ValueError(f"traces must have shape {want}, got {tuple(t.shape)}")
        return t

    # ----------------------------------------------------------- operators --
    def load_traces(self, traces: torch.Tensor, trace_major: bool = False) -> None:
        t = self._traces(traces, trace_major)
        _lib.check(self._lib.pstm_load_traces(self._handle, _ptr(t), int(trace_major),
                                              _stream_handle()))
        self._loaded_ref = t  # keep the source alive until the staging kernel ran

    def migrate_loaded(self, velocity, image: Optional[torch.Tensor] = None,
                       fold: Optional[torch.Tensor] = None, with_fold: bool = True):
        v, st, sc = self._vel(velocity)
        shape = (self.n_times, self.n_il, self.n_xl)
        if image is None:
            image = torch.empty(shape, device=self.device, dtype=torch.float32)
        if with_fold and fold is None:
            fold = torch.empty(shape, device=self.device, dtype=torch.float32)
        _lib.check(self._lib.pstm_migrate_loaded(self._handle, _ptr(v), st, sc, _ptr(image),
                                                 _ptr(fold) if with_fold else None,
                                                 _stream_handle()))
        return image, fold

    def migrate(self, traces: torch.Tensor, velocity, trace_major: bool = False,
                with_fold: bool = True):
        """Forward migration (data -> image, fold), the work of migrate_kirchhoff_full."""
        self.load_traces(traces, trace_major)
        return self.migrate_loaded(velocity, with_fold=with_fold)

    def fold(self, velocity) -> torch.Tensor:
        v, st, sc = self._vel(velocity)
        out = torch.empty((self.n_times, self.n_il, self.n_xl), device=self.device,
                          dtype=torch.float32)
        _lib.check(self._lib.pstm_fold(self._handle, _ptr(v), st, sc, _ptr(out), _stream_handle()))
        return out

    def demigrate(self, image: torch.Tensor, velocity, trace_major: bool = False) -> torch.Tensor:
        """Adjoint (image -> data): Kirchhoff demigration, the transpose of ``migrate``."""
        img = image.to(self.device, torch.float32).contiguous()
        if img.numel() != self.n_times * self.n_cols:
            raise ValueError("image must have n_times * n_il * n_xl elements")
        v, st, sc = self._vel(velocity)
        shape = (self.n_traces, self.n_samples) if trace_major else (self.n_samples, self.n_traces)
        out = torch.empty(shape, device=self.device, dtype=torch.float32)
        _lib.check(self._lib.pstm_demigrate(self._handle, _ptr(img), _ptr(v), st, sc, _ptr(out),
                                            int(trace_major), _stream_handle()))
        return out

    def velocity_gradient(self, grad_image: torch.Tensor, velocity) -> torch.Tensor:
        """d<grad_image, migrate(loaded traces; V)>/dV at every output sample."""
        g = grad_image.to(self.device, torch.float32).contiguous()
        v, st, sc = self._vel(velocity)
        out = torch.empty((self.n_times, self.n_il, self.n_xl), device=self.device,
                          dtype=torch.float32)
        _lib.check(self._lib.pstm_velocity_gradient(self._handle, _ptr(g), _ptr(v), st, sc,
                                                    _ptr(out), _stream_handle()))
        return out


def normalize_by_fold(image: torch.Tensor, fold: torch.Tensor, min_fold: int = 1) -> torch.Tensor:
    """image / fold where fold >= min_fold, else unchanged (new tensor)."""
    if image.shape != fold.shape:
        raise ValueError("image and fold must have the same shape")
    require_cuda()
    dev = image.device if image.is_cuda else torch.device("cuda")
    img = image.to(dev, torch.float32).contiguous()
    fd = fold.to(dev, torch.float32).contiguous()
    out = torch.empty_like(img)
    _lib.check(_lib.lib().pstm_normalize_by_fold(_ptr(img), _ptr(fd), _ptr(out), img.numel(),
                                                 float(min_fold), _stream_handle()))
    return out.to(image.device)


def normalize_mute(image: torch.Tensor, fold: torch.Tensor, min_fold: int = 1) -> torch.Tensor:
    """image / max(fold, min_fold), zero where fold < min_fold (migrate_dataset
    and MigrationResult.apply_fold_normalization semantics)."""
    require_cuda()
    dev = image.device if image.is_cuda else torch.device("cuda")
    img = image.to(dev, torch.float32).contiguous()
    fd = fold.to(dev, torch.float32).contiguous()
    out = torch.empty_like(img)
    _lib.check(_lib.lib().pstm_normalize_mute(_ptr(img), _ptr(fd), _ptr(out), img.numel(),
                                              float(min_fold), _stream_handle()))
    return out.to(image.device)


def regular_grid_from_points(output_x: np.ndarray, output_y: np.ndarray, n_il: int,
                             n_xl: int) -> Tuple[float, float, float, float, float, float]:
    """(origin_x, origin_y, il_dx, il_dy, xl_dx, xl_dy) of il-major output points;
    raises ValueError if the points are not a regular (possibly rotated) grid."""
    x = np.asarray(output_x, np.float64).reshape(n_il, n_xl)
    y = np.asarray(output_y, np.float64).reshape(n_il, n_xl)
    ox, oy = x[0, 0], y[0, 0]
    il_dx = (x[-1, 0] - ox) / (n_il - 1) if n_il > 1 else 0.0
    il_dy = (y[-1, 0] - oy) / (n_il - 1) if n_il > 1 else 0.0
    xl_dx = (x[0, -1] - ox) / (n_xl - 1) if n_xl > 1 else 0.0
    xl_dy = (y[0, -1] - oy) / (n_xl - 1) if n_xl > 1 else 0.0
    il = np.arange(n_il)[:, None]
    xl = np.arange(n_xl)[None, :]
    ex = ox + il * il_dx + xl * xl_dx
    ey = oy + il * il_dy + xl * xl_dy
    scale = max(1.0, np.abs(x).max(), np.abs(y).max())
    if np.abs(ex - x).max() > 1e-5 * scale or np.abs(ey - y).max() > 1e-5 * scale:
        raise ValueError("output points must form a regular il-major grid")
    return ox, oy, il_dx, il_dy, xl_dx, xl_dy


def regular_times_from_depth(depth_axis: np.ndarray, velocity: float) -> Tuple[float, float]:
    """(t0_ms, dt_ms) of the output times t = 2000 z / V of a depth axis."""
    z = np.asarray(depth_axis, np.float64)
    t = 2000.0 * z / float(velocity)
    n = t.shape[0]
    dt = (t[-1] - t[0]) / (n - 1) if n > 1 else 1.0
    if n > 1 and np.abs(t - (t[0] + np.arange(n) * dt)).max() > 1e-4 * max(1.0, abs(dt) * n):
        raise ValueError("depth_axis must correspond to a regular output time axis")
    return float(t[0]), float(dt if dt > 0 else 1.0)


def migrate_kirchhoff_full(traces: torch.Tensor, source_x: torch.Tensor, source_y: torch.Tensor,
                           receiver_x: torch.Tensor, receiver_y: torch.Tensor,
                           output_x: torch.Tensor, output_y: torch.Tensor,
                           depth_axis: torch.Tensor, velocity: Union[float, torch.Tensor],
                           dt_ms: float, t_min_ms: float, max_aperture_m: float,
                           max_angle_deg: float, n_il: int, n_xl: int,
                           progress_callback: Optional[Callable[[float, str], None]] = None,
                           enable_profiling: bool = False,
                           use_time_dependent_aperture: bool = False,
                           kernel_backend=None, storage: str = "f32", variant: int = 0,
                           out_t0_ms: Optional[float] = None, out_dt_ms: Optional[float] = None,
                           ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Full Kirchhoff migration, output-point centric, on the sm_100a kernels.

    Same arguments and results as the reference: traces (n_samples, n_traces),
    coordinates (n_traces,), output points (n_il*n_xl,) il-major, depth axis
    z = V t / 2 (n_depths,); returns image and fold (n_depths, n_il, n_xl).
    ``velocity`` may also be a V_rms tensor of shape (n_depths,) or
    (n_depths, n_il, n_xl); then pass the output time axis as ``out_t0_ms`` /
    ``out_dt_ms`` (the depth axis is ignored).
    """
    t_start = time.perf_counter()
    require_cuda(kernel_backend)
    in_dev = traces.device
    n_s, n_tr = traces.shape
    n_d = int(depth_axis.shape[0])
    ox, oy, ildx, ildy, xldx, xldy = regular_grid_from_points(
        torch.as_tensor(output_x).cpu().numpy(), torch.as_tensor(output_y).cpu().numpy(), n_il, n_xl)
    if torch.is_tensor(velocity) and velocity.numel() > 1:
        if out_t0_ms is None or out_dt_ms is None:
            raise ValueError("a V_rms tensor needs out_t0_ms and out_dt_ms")
        t0, dto = out_t0_ms, out_dt_ms
        vel = velocity
    else:
        vscal = float(velocity)
        z = torch.as_tensor(depth_axis).cpu().numpy().astype(np.float64)
        # migrate_bin_full builds the depth axis from the trace time axis
        # (migration_engine.py:305-306); recognise it to keep t0/dt exact
        tk = np.arange(n_d, dtype=np.float32) * np.float32(dt_ms) + np.float32(t_min_ms)
        zk = np.float32(vscal) * (tk / np.float32(1000.0)) / np.float32(2.0)
        if n_d and np.allclose(zk, z, rtol=1e-5, atol=1e-3):
            t0, dto = float(t_min_ms), float(dt_ms)
        else:
            t0, dto = regular_times_from_depth(z, vscal)
        if out_t0_ms is not None:
            t0 = out_t0_ms
        if out_dt_ms is not None:
            dto = out_dt_ms
        vel = torch.tensor([vscal], dtype=torch.float32)
    if progress_callback:
        progress_callback(0.0, "Building migration plan")
    plan = PSTMPlan(source_x, source_y, receiver_x, receiver_y, n_il=n_il, n_xl=n_xl, n_times=n_d,
                    origin_x=ox, origin_y=oy, il_dx=ildx, il_dy=ildy, xl_dx=xldx, xl_dy=xldy,
                    t0_ms=t0, dt_ms=dto, n_samples=n_s, in_t0_ms=t_min_ms, in_dt_ms=dt_ms,
                    max_aperture_m=max_aperture_m, max_angle_deg=max_angle_deg,
                    time_dependent_aperture=use_time_dependent_aperture, storage=storage,
                    variant=variant, kernel_backend=kernel_backend, forward_only=True)
    try:
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)] if enable_profiling else None
        if ev:
            ev[0].record()
        image, fold = plan.migrate(traces, vel)
        if ev:
            ev[1].record()
        plan.check()
        if ev:
            pairs = float(fold.double().sum().item())
            ms = ev[0].elapsed_time(ev[1])
            logger.info("PSTM kernel: %.2f ms, %.3e pairs, %.2f Gpairs/s, plan %s", ms, pairs,
                        pairs / ms / 1e6 if ms > 0 else float("nan"), plan.stats())
    finally:
        plan.close()
    if progress_callback:
        el = time.perf_counter() - t_start
        progress_callback(1.0, f"Migrated {n_il * n_xl} output points x {n_d} samples "
                               f"in {el:.2f}s")
    return image.to(in_dev), fold.to(in_dev)
