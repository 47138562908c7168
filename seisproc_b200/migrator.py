"""BaseMigrator API on the sm_100a kernels.

Keeps the reference's migrator interface (processors/migration/base_migrator.py:24-386,
kirchhoff_migrator.py:40-592):

* ``BaseMigrator(velocity_model, config)`` with ``migrate_gather``,
  ``migrate_dataset``, ``estimate_memory_gb``, progress callbacks
  ``(current, total, message)``, ``get_status``/``to_dict``;
* ``KirchhoffMigrator(velocity, config, device=None, use_traveltime_lut=True)``:
  ``migrate_gather(gather, geometry, output_image=None, output_fold=None)``
  accumulates into the passed tensors and returns them; the direct-DSR branch
  of ``_migrate_chunk`` (:362-402) is what the kernel computes -- trace time
  origin 0, sample index clamped to [0, n_samples - 2], angle mask
  atan2(h, |z| + 1e-6) < theta, per-leg aperture;
* ``MigrationResult`` with ``apply_fold_normalization`` (:317-349).

Velocity and traveltimes as the reference: v0 of the model, depth z = v0 t / 2,
straight rays, or (``use_traveltime_lut=True``, the default) the curved rays of
its traveltime table when the model has a v(z) gradient -- computed exactly
where the reference interpolates a bilinear (h, z) table
(traveltime_lut.py:141-167, 250-308; the images agree to ~1e-5).

Differences, each deliberate: ``config.weight_mode`` is honoured (SPREADING is
the reference's 1/(r_s r_r + 1e-6); FULL is obliquity x spreading; OBLIQUITY and
NONE as named) and ``min_offset_m``/``max_offset_m`` select the traces; a
laterally varying velocity model (which the reference cannot migrate with), or
any model with ``vrms_velocity=True``, is used as V_rms(t0, x, y).
"""
from __future__ import annotations

import logging
import time
from abc import ABC, abstractmethod
from typing import Any, Callable, Dict, List, Optional, Tuple

import numpy as np
import torch

from .kernel_backend import require_cuda
from .models import (MigrationConfig, MigrationGeometry, SeismicData, VelocityModel,
                     VelocityType, WeightMode)

logger = logging.getLogger(__name__)

ProgressCallback = Callable[[int, int, str], None]

_WEIGHT_OF_MODE = {WeightMode.SPREADING: "spreading", WeightMode.FULL: "obliquity_spreading",
                   WeightMode.OBLIQUITY: "obliquity", WeightMode.NONE: "none"}


class BaseMigrator(ABC):
    def __init__(self, velocity_model: VelocityModel, config: MigrationConfig, **kwargs):
        self.velocity_model = velocity_model
        self.config = config
        self.params = kwargs
        self._progress_callback: Optional[ProgressCallback] = None
        self._validate_inputs()

    @abstractmethod
    def _validate_inputs(self):
        ...

    def set_progress_callback(self, callback: Optional[ProgressCallback]) -> "BaseMigrator":
        self._progress_callback = callback
        return self

    def _report_progress(self, current: int, total: int, message: str = ""):
        if self._progress_callback is not None:
            self._progress_callback(current, total, message)

    @abstractmethod
    def migrate_gather(self, gather: SeismicData, geometry: MigrationGeometry):
        ...

    @abstractmethod
    def migrate_dataset(self, gathers: List[SeismicData], geometries: List[MigrationGeometry],
                        batch_size: int = 1) -> "MigrationResult":
        ...

    @abstractmethod
    def estimate_memory_gb(self, n_traces: int, n_samples: int) -> float:
        ...

    def can_process(self, n_traces: int, n_samples: int, available_memory_gb: float) -> bool:
        return self.estimate_memory_gb(n_traces, n_samples) < available_memory_gb * 0.8

    def calculate_batch_size(self, n_traces_per_gather: int, n_samples: int,
                             available_memory_gb: float) -> int:
        per = self.estimate_memory_gb(n_traces_per_gather, n_samples)
        if per <= 0:
            return 1
        return max(1, int(available_memory_gb * 0.7 / per))

    @abstractmethod
    def get_description(self) -> str:
        ...

    def get_status(self) -> Dict[str, Any]:
        g = self.config.output_grid
        return {"class": self.__class__.__name__,
                "velocity_type": str(self.velocity_model.velocity_type),
                "output_grid": f"{g.n_inline}x{g.n_xline}x{g.n_time}",
                "max_aperture": self.config.max_aperture_m,
                "max_angle": self.config.max_angle_deg}

    def to_dict(self) -> Dict[str, Any]:
        return {"class_name": self.__class__.__name__, "module": self.__class__.__module__,
                "velocity_model": self.velocity_model.to_dict(),
                "config": self.config.to_dict(), "params": self.params}


class MigrationResult:
    """Migrated image (n_time, n_inline, n_xline) float32, fold int32, metadata."""

    def __init__(self, image: np.ndarray, fold: Optional[np.ndarray] = None,
                 config: Optional[MigrationConfig] = None,
                 metadata: Optional[Dict[str, Any]] = None):
        self.image = np.asarray(image).astype(np.float32)
        self.fold = np.asarray(fold).astype(np.int32) if fold is not None else None
        self.config = config
        self.metadata = metadata or {}

    @property
    def shape(self):
        return self.image.shape

    @property
    def n_time(self) -> int:
        return self.image.shape[0]

    @property
    def n_inline(self) -> int:
        return self.image.shape[1]

    @property
    def n_xline(self) -> int:
        return self.image.shape[2]

    def get_inline_section(self, xline_idx: int) -> np.ndarray:
        return self.image[:, :, xline_idx]

    def get_xline_section(self, inline_idx: int) -> np.ndarray:
        return self.image[:, inline_idx, :]

    def get_time_slice(self, time_idx: int) -> np.ndarray:
        return self.image[time_idx, :, :]

    def apply_fold_normalization(self, min_fold: int = 1) -> "MigrationResult":
        if self.fold is None:
            return self
        out = self.image / np.maximum(self.fold, min_fold)
        out[self.fold < min_fold] = 0.0
        return MigrationResult(out, self.fold.copy(), self.config,
                               {**self.metadata, "fold_normalized": True, "min_fold": min_fold})

    def get_statistics(self) -> Dict[str, Any]:
        f = self.fold
        return {"shape": self.shape, "image_min": float(np.min(self.image)),
                "image_max": float(np.max(self.image)), "image_mean": float(np.mean(self.image)),
                "image_std": float(np.std(self.image)),
                "image_rms": float(np.sqrt(np.mean(self.image ** 2))),
                "fold_min": int(np.min(f)) if f is not None else None,
                "fold_max": int(np.max(f)) if f is not None else None,
                "fold_mean": float(np.mean(f)) if f is not None else None}


def offset_taper(offset: np.ndarray, min_offset: float, max_offset: float,
                 taper_width: float) -> np.ndarray:
    """Per-trace weight of the aperture controller's offset mask
    (processors/migration/aperture.py:197-226): 0 outside [min, max], a cosine
    rise over the first ``taper_width`` of the range and a fall over the last."""
    o = np.asarray(offset, np.float64)
    span = taper_width * (max_offset - min_offset)
    w = ((o >= min_offset) & (o <= max_offset)).astype(np.float64)
    if span > 0:
        rise = (o >= min_offset) & (o < min_offset + span)
        w = np.where(rise, w * 0.5 * (1.0 - np.cos(np.pi * (o - min_offset) / span)), w)
        fall = (o > max_offset - span) & (o <= max_offset)
        w = np.where(fall, w * 0.5 * (1.0 + np.cos(np.pi * (o - max_offset + span) / span)), w)
    return w


class KirchhoffMigrator(BaseMigrator):
    """Output-driven Kirchhoff PSTM on the CUDA sm_100a kernels."""

    def __init__(self, velocity: VelocityModel, config: MigrationConfig,
                 device: Optional[torch.device] = None, use_traveltime_lut: bool = True,
                 kernel_backend=None, storage: str = "f32", variant: int = 0,
                 antialias: bool = False, aa_max_halfwidth: float = 32.0,
                 aperture_taper: bool = False, vrms_velocity: bool = False):
        self.velocity = velocity
        require_cuda(kernel_backend)
        self.device = torch.device(device) if device is not None else \
            torch.device("cuda", torch.cuda.current_device())
        if self.device.type != "cuda":
            raise ValueError("KirchhoffMigrator runs on a CUDA device only")
        # The reference's velocity semantics: v0 for every model, z = v0 t / 2,
        # straight rays; with its default traveltime table a v(z) gradient turns
        # the rays into arcs (computed exactly here, not interpolated from a
        # table).  vrms_velocity=True takes the model as V_rms(t0, x, y) instead.
        self._use_traveltime_lut = use_traveltime_lut
        self.vrms_velocity = vrms_velocity
        self.kernel_backend = kernel_backend
        self.storage = storage
        self.variant = variant
        # the reference migrator never applies its anti-alias filter; it is an
        # explicit opt-in here (weight FULL only)
        self.antialias = antialias
        self.aa_max_halfwidth = aa_max_halfwidth
        # likewise the aperture controller's cosine tapers (config.taper_width:
        # offset per trace, distance and angle per leg), float32 storage only
        self.aperture_taper = aperture_taper
        super().__init__(velocity, config)

    def _validate_inputs(self):
        if self.velocity.v0 is None or self.velocity.v0 <= 0:
            raise ValueError("Velocity model must have positive v0")
        if self.config.output_grid.n_time <= 0:
            raise ValueError("Output grid must have positive n_time")

    def _columns(self) -> Tuple[np.ndarray, np.ndarray]:
        g = self.config.output_grid
        il = np.arange(g.n_inline)[:, None]
        xl = np.arange(g.n_xline)[None, :]
        x = (g.x_origin + il * g.d_inline + 0 * xl).ravel()
        y = (g.y_origin + 0 * il + xl * g.d_xline).ravel()
        return x, y

    def _velocity_and_rays(self) -> Tuple[torch.Tensor, float]:
        """(velocity on the device, ray gradient k) of a migration.  The
        reference migrator uses v0 alone (kirchhoff_migrator.py:312,
        migrate_gather :221-224); its default traveltime table bends the rays
        when the model has a gradient (:146-175, traveltime_lut.py:141-167).
        Laterally varying models (the reference cannot migrate with them) and
        ``vrms_velocity`` use the model as V_rms at every output sample."""
        vm = self.velocity
        lateral = vm.velocity_type in (VelocityType.V_OF_XZ, VelocityType.V_OF_XYZ)
        if self.vrms_velocity or lateral or vm.v0 is None:
            return self._velocity_grid(), 0.0
        k = float(vm.gradient or 0.0) if self._use_traveltime_lut else 0.0
        if abs(k) < 1e-10:
            k = 0.0
        return torch.full((1,), float(vm.v0), dtype=torch.float32, device=self.device), k

    def _velocity_grid(self) -> torch.Tensor:
        """V at the output samples on the device (laterally varying models are
        resampled there by ``velocity_io.velocity_grid``)."""
        from .velocity_io import velocity_grid
        g = self.config.output_grid
        if self.velocity.is_constant:
            return torch.full((1,), float(self.velocity.v0), dtype=torch.float32,
                              device=self.device)
        cx, cy = self._columns()
        return velocity_grid(self.velocity, g.time_axis, cx, cy, self.device)

    def migrate_gather(self, gather: SeismicData, geometry: MigrationGeometry,
                       output_image: Optional[torch.Tensor] = None,
                       output_fold: Optional[torch.Tensor] = None):
        from .kirchhoff import PSTMPlan
        g = self.config.output_grid
        shape = (g.n_time, g.n_inline, g.n_xline)
        if output_image is None:
            output_image = torch.zeros(shape, device=self.device, dtype=torch.float32)
        if output_fold is None:
            output_fold = torch.zeros(shape, device=self.device, dtype=torch.float32)
        off = geometry.offset
        sel = np.nonzero((off >= self.config.min_offset_m) &
                         (off <= self.config.max_offset_m))[0]
        if sel.size == 0:
            return output_image, output_fold
        full = sel.size == geometry.n_traces
        traces = gather.traces if full else gather.traces[:, sel]
        tw = float(self.config.taper_width) if self.aperture_taper else 0.0
        v, ray_k = self._velocity_and_rays()
        if tw > 0 and ray_k != 0:
            raise NotImplementedError(
                "aperture tapers with curved rays are not built: pass use_traveltime_lut=False "
                "(straight rays at v0) or vrms_velocity=True")
        if tw > 0:
            w_off = offset_taper(off[sel], self.config.min_offset_m, self.config.max_offset_m, tw)
            traces = np.asarray(traces, np.float32) * w_off[None, :].astype(np.float32)
        coords = [a if full else a[sel] for a in (geometry.source_x, geometry.source_y,
                                                  geometry.receiver_x, geometry.receiver_y)]
        with torch.cuda.device(self.device):
            plan = PSTMPlan(
                *[torch.from_numpy(np.ascontiguousarray(a)).to(self.device) for a in coords],
                n_il=g.n_inline, n_xl=g.n_xline, n_times=g.n_time, origin_x=g.x_origin,
                origin_y=g.y_origin, il_dx=g.d_inline, il_dy=0.0, xl_dx=0.0, xl_dy=g.d_xline,
                t0_ms=g.t0 * 1000.0, dt_ms=g.dt * 1000.0, n_samples=traces.shape[0],
                in_t0_ms=0.0, in_dt_ms=float(gather.sample_rate),
                max_aperture_m=self.config.max_aperture_m,
                max_angle_deg=self.config.max_angle_deg,
                weight=_WEIGHT_OF_MODE[self.config.weight_mode], clamp="migrator",
                storage=self.storage, variant=self.variant, kernel_backend=self.kernel_backend,
                antialias=self.antialias, aa_dx=g.d_inline, aa_dy=g.d_xline,
                aa_max_halfwidth=self.aa_max_halfwidth, forward_only=True, taper_width=tw,
                ray_gradient=ray_k)
            try:
                tr = torch.from_numpy(np.ascontiguousarray(traces, dtype=np.float32))
                img, fold = plan.migrate(tr.to(self.device), v)
                plan.check()
            finally:
                plan.close()
            output_image += img
            output_fold += fold
        return output_image, output_fold

    def migrate_dataset(self, gathers: List[SeismicData], geometries: List[MigrationGeometry],
                        progress_callback: Optional[Callable[[float, str], None]] = None,
                        batch_size: int = 1) -> MigrationResult:
        from .kirchhoff import normalize_mute
        t0 = time.time()
        g = self.config.output_grid
        shape = (g.n_time, g.n_inline, g.n_xline)
        image = torch.zeros(shape, device=self.device, dtype=torch.float32)
        fold = torch.zeros(shape, device=self.device, dtype=torch.float32)
        n = len(gathers)
        for i, (ga, ge) in enumerate(zip(gathers, geometries)):
            if progress_callback:
                progress_callback(i / max(n, 1) * 100, f"Migrating gather {i + 1}/{n}")
            self._report_progress(i, n, f"Migrating gather {i + 1}/{n}")
            image, fold = self.migrate_gather(ga, ge, image, fold)
        if self.config.normalize_by_fold:
            image = normalize_mute(image, fold, self.config.min_fold)
        el = time.time() - t0
        if progress_callback:
            progress_callback(100.0, "Migration complete")
        return MigrationResult(image.cpu().numpy(), fold.cpu().numpy(), self.config,
                               {"n_gathers": n, "elapsed_seconds": el,
                                "traces_per_second": sum(x.n_traces for x in gathers) / max(el, 1e-9),
                                "velocity_v0": self.velocity.v0})

    def estimate_memory_gb(self, n_traces: int, n_samples: int) -> float:
        g = self.config.output_grid
        out = 2 * g.total_samples * 4
        data = n_traces * (n_samples + 8) * 4 * 2 + n_traces * 64
        return (out + data) / 1024 ** 3

    def get_description(self) -> str:
        return (f"Kirchhoff PSTM (CUDA sm_100a), v0={self.velocity.v0:.0f} m/s, "
                f"aperture={self.config.max_aperture_m:.0f} m, "
                f"angle={self.config.max_angle_deg:.0f} deg, "
                f"weight={self.config.weight_mode.value}")


def create_kirchhoff_migrator(velocity: VelocityModel, config: MigrationConfig,
                              device: Optional[torch.device] = None, **kw) -> KirchhoffMigrator:
    return KirchhoffMigrator(velocity, config, device=device, **kw)
