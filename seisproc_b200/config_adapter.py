"""Wizard configuration -> MigrationEngine.migrate_bin_full arguments.

Same keys, fallbacks and validation messages as the reference adapter
(processors/migration/config_adapter.py:21-395).  Two keys are added for the
B200 engine: ``velocity_model`` (a V_rms model passed straight through) and
``kernel_backend``.
"""
from __future__ import annotations

import logging
from dataclasses import dataclass
from typing import Any, Callable, Dict, Optional, Tuple

import numpy as np

logger = logging.getLogger(__name__)


@dataclass
class MigrationParams:
    origin_x: float
    origin_y: float
    il_spacing: float
    xl_spacing: float
    azimuth_deg: float
    n_il: int
    n_xl: int
    dt_ms: float
    t_min_ms: float
    n_samples: int
    velocity_mps: float
    max_aperture_m: float
    max_angle_deg: float
    tile_size: int = 100
    use_time_domain: bool = False
    use_kdtree: bool = False
    sample_batch_size: int = 200
    max_traces_per_tile: int = 5000


class ConfigAdapter:
    """Maps PSTM wizard keys (x_origin, output_bin_il, inline_min/max/step, ...)
    onto the engine's parameters."""

    def __init__(self, config: Dict[str, Any]):
        self.config = config
        self._params: Optional[MigrationParams] = None

    @property
    def params(self) -> MigrationParams:
        if self._params is None:
            self._params = self._extract_params()
        return self._params

    def _extract_params(self) -> MigrationParams:
        c = self.config
        il_sp = c.get("output_bin_il", c.get("input_bin_il", 25.0))
        xl_sp = c.get("output_bin_xl", c.get("input_bin_xl", 25.0))
        n_il = max(1, (c.get("inline_max", 100) - c.get("inline_min", 1)) // c.get("inline_step", 1) + 1)
        n_xl = max(1, (c.get("xline_max", 100) - c.get("xline_min", 1)) // c.get("xline_step", 1) + 1)
        dt = c.get("dt_ms", 4.0)
        if dt <= 0:
            dt = 4.0
        t0 = c.get("time_min_ms", 0.0)
        n_s = max(1, int((c.get("time_max_ms", 6000.0) - t0) / dt) + 1)
        return MigrationParams(
            origin_x=c.get("x_origin", 0.0), origin_y=c.get("y_origin", 0.0), il_spacing=il_sp,
            xl_spacing=xl_sp, azimuth_deg=c.get("grid_azimuth_deg", 0.0), n_il=n_il, n_xl=n_xl,
            dt_ms=dt, t_min_ms=t0, n_samples=n_s, velocity_mps=c.get("velocity_v0", 2500.0),
            max_aperture_m=c.get("max_aperture_m", 5000.0),
            max_angle_deg=c.get("max_angle_deg", 60.0), tile_size=c.get("tile_size", 100),
            use_time_domain=c.get("use_time_domain", False), use_kdtree=c.get("use_kdtree", False),
            sample_batch_size=c.get("sample_batch_size", 200),
            max_traces_per_tile=c.get("max_traces_per_tile", 5000))

    def get_engine_params(self, traces: np.ndarray, source_x: np.ndarray, source_y: np.ndarray,
                          receiver_x: np.ndarray, receiver_y: np.ndarray, normalize: bool = True,
                          min_fold: int = 1,
                          progress_callback: Optional[Callable[[float, str], None]] = None,
                          enable_profiling: bool = False,
                          use_time_dependent_aperture: bool = False) -> Dict[str, Any]:
        """kwargs for MigrationEngine.migrate_bin_full()."""
        p = self.params
        out = {
            "traces": traces, "source_x": source_x, "source_y": source_y,
            "receiver_x": receiver_x, "receiver_y": receiver_y,
            "origin_x": p.origin_x, "origin_y": p.origin_y, "il_spacing": p.il_spacing,
            "xl_spacing": p.xl_spacing, "azimuth_deg": p.azimuth_deg, "n_il": p.n_il,
            "n_xl": p.n_xl, "dt_ms": p.dt_ms, "t_min_ms": p.t_min_ms, "n_times": p.n_samples,
            "velocity_mps": p.velocity_mps, "max_aperture_m": p.max_aperture_m,
            "max_angle_deg": p.max_angle_deg, "normalize": normalize, "min_fold": min_fold,
            "progress_callback": progress_callback, "enable_profiling": enable_profiling,
            "use_time_dependent_aperture": use_time_dependent_aperture,
        }
        if self.config.get("velocity_model") is not None:
            out["velocity_model"] = self.config["velocity_model"]
        if self.config.get("kernel_backend") is not None:
            out["kernel_backend"] = self.config["kernel_backend"]
        return out

    def get_time_domain_params(self, traces: np.ndarray, source_x: np.ndarray,
                               source_y: np.ndarray, receiver_x: np.ndarray,
                               receiver_y: np.ndarray, normalize: bool = True, min_fold: int = 1,
                               progress_callback: Optional[Callable[[float, str], None]] = None,
                               enable_profiling: bool = False,
                               use_time_dependent_aperture: bool = True) -> Dict[str, Any]:
        """The reference's kwargs for the time-domain entries
        (config_adapter.py:239-304): the engine arguments with ``tile_size``
        and a time-dependent aperture by default.  The batch worker takes the
        grid keys from it for ``migrate_bin_time_domain_rms``
        (views/migration_monitor_dialog.py:288-362), adding ``velocity_model``,
        ``n_times`` and the params' ``tile_size``, ``sample_batch_size`` and
        ``max_traces_per_tile``."""
        p = self.params
        return {
            "traces": traces, "source_x": source_x, "source_y": source_y,
            "receiver_x": receiver_x, "receiver_y": receiver_y,
            "origin_x": p.origin_x, "origin_y": p.origin_y, "il_spacing": p.il_spacing,
            "xl_spacing": p.xl_spacing, "azimuth_deg": p.azimuth_deg, "n_il": p.n_il,
            "n_xl": p.n_xl, "dt_ms": p.dt_ms, "t_min_ms": p.t_min_ms, "n_times": p.n_samples,
            "velocity_mps": p.velocity_mps, "max_aperture_m": p.max_aperture_m,
            "max_angle_deg": p.max_angle_deg, "tile_size": p.tile_size,
            "normalize": normalize, "min_fold": min_fold,
            "progress_callback": progress_callback, "enable_profiling": enable_profiling,
            "use_time_dependent_aperture": use_time_dependent_aperture,
        }

    def validate(self) -> Tuple[bool, str]:
        issues = []
        c = self.config
        if c.get("dt_ms", 4.0) <= 0:
            issues.append(f"Invalid sample interval: {c.get('dt_ms')}ms")
        if c.get("inline_max", 100) < c.get("inline_min", 1):
            issues.append(f"Invalid inline range: max ({c.get('inline_max')}) < min "
                          f"({c.get('inline_min')})")
        if c.get("xline_max", 100) < c.get("xline_min", 1):
            issues.append(f"Invalid crossline range: max ({c.get('xline_max')}) < min "
                          f"({c.get('xline_min')})")
        p = self.params
        if p.n_il <= 0:
            issues.append(f"Invalid inline count: {p.n_il}")
        if p.n_xl <= 0:
            issues.append(f"Invalid crossline count: {p.n_xl}")
        if p.n_il * p.n_xl > 1e8:
            issues.append(f"Grid too large: {p.n_il}x{p.n_xl} = {p.n_il * p.n_xl:.0e} points")
        if p.n_samples <= 0:
            issues.append(f"Invalid sample count: {p.n_samples}")
        if p.velocity_mps <= 0:
            issues.append(f"Invalid velocity: {p.velocity_mps} m/s")
        elif p.velocity_mps < 1000 or p.velocity_mps > 8000:
            issues.append(f"Unusual velocity: {p.velocity_mps} m/s (typical range: 1000-8000)")
        if p.max_aperture_m <= 0:
            issues.append(f"Invalid aperture: {p.max_aperture_m}m")
        if p.max_angle_deg <= 0 or p.max_angle_deg > 90:
            issues.append(f"Invalid max angle: {p.max_angle_deg}°")
        if issues:
            return False, "; ".join(issues)
        return True, "Configuration valid"

    def get_summary(self) -> str:
        p = self.params
        return "\n".join([
            "Migration Parameters:",
            f"  Output grid: {p.n_il} IL x {p.n_xl} XL",
            f"  Origin: ({p.origin_x:.1f}, {p.origin_y:.1f})",
            f"  Bin sizes: {p.il_spacing:.1f}m IL, {p.xl_spacing:.1f}m XL",
            f"  Azimuth: {p.azimuth_deg:.1f}°",
            f"  Time: {p.t_min_ms:.0f} - {p.t_min_ms + (p.n_samples - 1) * p.dt_ms:.0f} ms "
            f"@ {p.dt_ms:.1f}ms",
            f"  Velocity: {p.velocity_mps:.0f} m/s",
            f"  Aperture: {p.max_aperture_m:.0f}m, angle: {p.max_angle_deg:.0f}°",
        ])


def create_adapter_from_wizard(config: Dict[str, Any]) -> ConfigAdapter:
    return ConfigAdapter(config)
