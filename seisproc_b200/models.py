"""Data models of the PSTM path: velocity, output grid / migration config,
survey geometry and seismic data.

These keep the reference's dataclass interfaces (field names, defaults,
validation errors) so callers can pass the same objects:

* ``VelocityType`` / ``VelocityModel``       models/velocity_model.py:22-363
* ``create_constant_velocity`` ... ``create_3d_velocity``,
  ``rms_to_interval_velocity`` / ``interval_to_rms_velocity`` (Dix)
                                              models/velocity_model.py:370-599
* ``TraveltimeMode`` / ``InterpolationMode`` / ``WeightMode`` / ``OutputGrid`` /
  ``MigrationConfig``                         models/migration_config.py:20-359
* ``MigrationGeometry``                       models/migration_geometry.py:19-402
* ``SeismicData``                             models/seismic_data.py:16-97

The velocity values are read as V_rms for time migration (``is_time`` axis in
two-way seconds).  ``VelocityModel.rms_grid`` samples a model at the output
points; it is host-side setup, run once per migration call.
"""
from __future__ import annotations

import logging
from dataclasses import dataclass, field
from enum import Enum
from typing import Any, Dict, Optional, Tuple, Union

import numpy as np

logger = logging.getLogger(__name__)


# ----------------------------------------------------------------- velocity --
class VelocityType(Enum):
    CONSTANT = "constant"
    V_OF_Z = "v_of_z"
    V_OF_XZ = "v_of_xz"
    V_OF_XYZ = "v_of_xyz"


def _interp_axis(ax: np.ndarray, q: np.ndarray):
    """Index and weight of linear interpolation along a monotone axis, with
    linear extrapolation beyond the ends (scipy RegularGridInterpolator with
    fill_value=None behaves this way)."""
    ax = np.asarray(ax, np.float64)
    q = np.asarray(q, np.float64)
    if ax.shape[0] == 1:
        return np.zeros(q.shape, np.int64), np.zeros(q.shape)
    i = np.clip(np.searchsorted(ax, q, side="right") - 1, 0, ax.shape[0] - 2)
    w = (q - ax[i]) / (ax[i + 1] - ax[i])
    return i, w


@dataclass
class VelocityModel:
    """Velocity model (constant, v(z), v(x,z) or v(x,y,z)); z is two-way time in
    seconds when ``is_time``.  Same fields as the reference model."""
    data: Union[float, np.ndarray]
    z_axis: Optional[np.ndarray] = None
    x_axis: Optional[np.ndarray] = None
    y_axis: Optional[np.ndarray] = None
    is_time: bool = True
    gradient: Optional[float] = None
    v0: Optional[float] = None
    metadata: Dict[str, Any] = field(default_factory=dict)

    def __post_init__(self):
        if isinstance(self.data, (int, float, np.floating)) and not isinstance(self.data, bool):
            self.data = float(self.data)
            self._type = VelocityType.CONSTANT
        elif isinstance(self.data, np.ndarray):
            nd = self.data.ndim
            if nd == 1:
                if self.z_axis is None:
                    raise ValueError("z_axis required for 1D velocity model")
                if len(self.z_axis) != len(self.data):
                    raise ValueError(f"z_axis length ({len(self.z_axis)}) must match data "
                                     f"length ({len(self.data)})")
                self._type = VelocityType.V_OF_Z
            elif nd == 2:
                if self.z_axis is None or self.x_axis is None:
                    raise ValueError("z_axis and x_axis required for 2D velocity model")
                self._type = VelocityType.V_OF_XZ
            elif nd == 3:
                if self.z_axis is None or self.x_axis is None or self.y_axis is None:
                    raise ValueError("z_axis, x_axis, y_axis required for 3D velocity model")
                self._type = VelocityType.V_OF_XYZ
            else:
                raise ValueError(f"Unsupported velocity data dimension: {nd}")
            self.data = self.data.astype(np.float32, copy=False)
        else:
            raise ValueError(f"Unsupported data type: {type(self.data)}")
        if self.v0 is None:
            if self._type == VelocityType.CONSTANT:
                self.v0 = self.data
            elif self._type == VelocityType.V_OF_Z:
                self.v0 = float(self.data[0]) if self.z_axis[0] == 0 else \
                    float(np.interp(0.0, self.z_axis, self.data))
        if self.gradient is None and self._type == VelocityType.V_OF_Z and len(self.z_axis) >= 2:
            self.gradient = float(np.polyfit(self.z_axis, self.data, 1)[0])
        self._validate()

    def _validate(self):
        lo = 0.1
        if self._type == VelocityType.CONSTANT:
            if self.data < lo:
                raise ValueError(f"Velocity must be >= {lo} m/s, got {self.data}")
        else:
            if np.min(self.data) < lo:
                logger.warning("clipping velocities below %s m/s", lo)
                self.data = np.clip(self.data, lo, None)

    @property
    def velocity_type(self) -> VelocityType:
        return self._type

    @property
    def is_constant(self) -> bool:
        return self._type == VelocityType.CONSTANT

    @property
    def has_gradient(self) -> bool:
        return self.gradient is not None and abs(self.gradient) > 1e-6

    def get_velocity_at(self, z, x=None, y=None):
        """Velocity at (z[, x[, y]]): linear / bilinear / trilinear interpolation."""
        if self._type == VelocityType.CONSTANT:
            if isinstance(z, np.ndarray):
                return np.full_like(z, self.data, dtype=np.float32)
            return self.data
        if self._type == VelocityType.V_OF_Z:
            return np.interp(z, self.z_axis, self.data).astype(np.float32)
        z = np.atleast_1d(np.asarray(z, np.float64))
        if x is None:
            raise ValueError("x coordinate required for 2D/3D velocity model")
        x = np.broadcast_to(np.atleast_1d(np.asarray(x, np.float64)), z.shape)
        iz, wz = _interp_axis(self.z_axis, z)
        ix, wx = _interp_axis(self.x_axis, x)
        d = self.data.astype(np.float64)
        nz1 = min(1, d.shape[0] - 1)
        nx1 = min(1, d.shape[1] - 1)
        if self._type == VelocityType.V_OF_XZ:
            v = ((1 - wz) * (1 - wx) * d[iz, ix] + wz * (1 - wx) * d[iz + nz1, ix] +
                 (1 - wz) * wx * d[iz, ix + nx1] + wz * wx * d[iz + nz1, ix + nx1])
            return v.astype(np.float32)
        if y is None:
            raise ValueError("x, y coordinates required for 3D velocity model")
        y = np.broadcast_to(np.atleast_1d(np.asarray(y, np.float64)), z.shape)
        iy, wy = _interp_axis(self.y_axis, y)
        ny1 = min(1, d.shape[2] - 1)
        v = 0.0
        for a, wa in ((0, 1 - wz), (nz1, wz)):
            for b, wb in ((0, 1 - wx), (nx1, wx)):
                for c, wc in ((0, 1 - wy), (ny1, wy)):
                    v = v + wa * wb * wc * d[iz + a, ix + b, iy + c]
        return np.asarray(v, dtype=np.float32)

    def rms_grid(self, t_s: np.ndarray, col_x: np.ndarray, col_y: np.ndarray) -> np.ndarray:
        """V at every output sample: (n_t,) for laterally invariant models,
        else (n_t, n_cols)."""
        t_s = np.asarray(t_s, np.float64)
        if self._type == VelocityType.CONSTANT:
            return np.full(1, self.data, np.float32)
        if self._type == VelocityType.V_OF_Z:
            return np.interp(t_s, self.z_axis, self.data).astype(np.float32)
        n_t, n_c = t_s.shape[0], col_x.shape[0]
        zz = np.repeat(t_s[:, None], n_c, 1)
        xx = np.repeat(np.asarray(col_x, np.float64)[None, :], n_t, 0)
        yy = np.repeat(np.asarray(col_y, np.float64)[None, :], n_t, 0)
        return self.get_velocity_at(zz.ravel(), xx.ravel(), yy.ravel()).reshape(n_t, n_c)

    def to_dict(self) -> Dict[str, Any]:
        out = {"velocity_type": self._type.value, "is_time": self.is_time,
               "gradient": self.gradient, "v0": self.v0, "metadata": dict(self.metadata)}
        if self._type == VelocityType.CONSTANT:
            out["data"] = self.data
        else:
            out["data"] = self.data.tolist()
            out["z_axis"] = np.asarray(self.z_axis).tolist()
            if self.x_axis is not None:
                out["x_axis"] = np.asarray(self.x_axis).tolist()
            if self.y_axis is not None:
                out["y_axis"] = np.asarray(self.y_axis).tolist()
        return out

    @classmethod
    def from_dict(cls, d: Dict[str, Any]) -> "VelocityModel":
        vt = VelocityType(d["velocity_type"])
        data = d["data"] if vt == VelocityType.CONSTANT else np.array(d["data"], np.float32)
        ax = lambda k: np.array(d[k]) if d.get(k) is not None else None
        return cls(data=data, z_axis=ax("z_axis"), x_axis=ax("x_axis"), y_axis=ax("y_axis"),
                   is_time=d.get("is_time", True), gradient=d.get("gradient"), v0=d.get("v0"),
                   metadata=d.get("metadata", {}))

    def copy(self) -> "VelocityModel":
        return VelocityModel.from_dict(self.to_dict())


def create_constant_velocity(velocity: float, is_time: bool = True) -> VelocityModel:
    return VelocityModel(data=float(velocity), is_time=is_time,
                         metadata={"model_type": "constant"})


def create_linear_gradient_velocity(v0: float, gradient: float, z_max: float, dz: float = 0.004,
                                    is_time: bool = True) -> VelocityModel:
    z = np.arange(0.0, z_max + dz / 2, dz, dtype=np.float32)
    return VelocityModel(data=(v0 + gradient * z).astype(np.float32), z_axis=z, is_time=is_time,
                         gradient=gradient, v0=v0, metadata={"model_type": "linear_gradient"})


def create_from_rms_velocity(t_axis: np.ndarray, v_rms: np.ndarray,
                             is_time: bool = True) -> VelocityModel:
    return VelocityModel(data=np.asarray(v_rms, np.float32), z_axis=np.asarray(t_axis, np.float32),
                         is_time=is_time, metadata={"model_type": "rms"})


def rms_to_interval_velocity(t_axis: np.ndarray, v_rms: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Dix: V_int(n)^2 = (V_rms(n)^2 t(n) - V_rms(n-1)^2 t(n-1)) / (t(n) - t(n-1))."""
    t = np.asarray(t_axis, np.float64)
    v = np.asarray(v_rms, np.float64)
    out = np.empty(t.shape[0], np.float32)
    out[0] = v[0]
    for i in range(1, t.shape[0]):
        dt = t[i] - t[i - 1]
        num = v[i] ** 2 * t[i] - v[i - 1] ** 2 * t[i - 1]
        out[i] = np.sqrt(num / dt) if (dt > 0 and num > 0) else v[i]
    return t_axis, out


def interval_to_rms_velocity(t_axis: np.ndarray, v_int: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """V_rms(n) = sqrt(sum V_int(i)^2 dt(i) / t(n))."""
    t = np.asarray(t_axis, np.float64)
    v = np.asarray(v_int, np.float64)
    out = np.empty(t.shape[0], np.float32)
    out[0] = v[0]
    acc = v[0] ** 2 * t[0] if t[0] > 0 else 0.0
    for i in range(1, t.shape[0]):
        acc += v[i] ** 2 * (t[i] - t[i - 1])
        out[i] = np.sqrt(acc / t[i]) if t[i] > 0 else v[i]
    return t_axis, out


def create_2d_velocity(data, z_axis, x_axis, is_time=True, metadata=None) -> VelocityModel:
    data = np.asarray(data, np.float32)
    if data.ndim != 2:
        raise ValueError(f"Data must be 2D, got shape {data.shape}")
    if data.shape != (len(z_axis), len(x_axis)):
        raise ValueError("data shape must be (len(z_axis), len(x_axis))")
    return VelocityModel(data=data, z_axis=np.asarray(z_axis, np.float32),
                         x_axis=np.asarray(x_axis, np.float32), is_time=is_time,
                         metadata=metadata or {"model_type": "2d_field"})


def create_3d_velocity(data, z_axis, x_axis, y_axis, is_time=True, metadata=None) -> VelocityModel:
    data = np.asarray(data, np.float32)
    if data.ndim != 3:
        raise ValueError(f"Data must be 3D, got shape {data.shape}")
    if data.shape != (len(z_axis), len(x_axis), len(y_axis)):
        raise ValueError("data shape must be (len(z_axis), len(x_axis), len(y_axis))")
    return VelocityModel(data=data, z_axis=np.asarray(z_axis, np.float32),
                         x_axis=np.asarray(x_axis, np.float32),
                         y_axis=np.asarray(y_axis, np.float32), is_time=is_time,
                         metadata=metadata or {"model_type": "3d_cube"})


# ----------------------------------------------------------- configuration --
class TraveltimeMode(Enum):
    STRAIGHT_RAY = "straight_ray"
    CURVED_RAY = "curved_ray"
    VTI = "vti"


class AnisotropyMethod(Enum):
    ANELLIPTIC = "anelliptic"
    EXACT = "exact"
    WEAK = "weak"


class InterpolationMode(Enum):
    LINEAR = "linear"
    SINC = "sinc"


class WeightMode(Enum):
    NONE = "none"
    SPREADING = "spreading"
    OBLIQUITY = "obliquity"
    FULL = "full"


@dataclass
class OutputGrid:
    """Output migration grid; ``dt`` and ``t0`` in seconds."""
    n_time: int = 1000
    n_inline: int = 100
    n_xline: int = 100
    dt: float = 0.004
    d_inline: float = 25.0
    d_xline: float = 25.0
    t0: float = 0.0
    inline_start: int = 1
    xline_start: int = 1
    x_origin: float = 0.0
    y_origin: float = 0.0
    inline_azimuth: float = 0.0

    def __post_init__(self):
        for name in ("n_time", "n_inline", "n_xline", "dt", "d_inline", "d_xline"):
            if getattr(self, name) <= 0:
                raise ValueError(f"{name} must be positive, got {getattr(self, name)}")

    @property
    def t_max(self) -> float:
        return self.t0 + (self.n_time - 1) * self.dt

    @property
    def time_axis(self) -> np.ndarray:
        return np.arange(self.n_time) * self.dt + self.t0

    @property
    def inline_axis(self) -> np.ndarray:
        return np.arange(self.n_inline) + self.inline_start

    @property
    def xline_axis(self) -> np.ndarray:
        return np.arange(self.n_xline) + self.xline_start

    @property
    def total_samples(self) -> int:
        return self.n_time * self.n_inline * self.n_xline

    @property
    def memory_gb(self) -> float:
        return self.total_samples * 4 / (1024 ** 3)

    def get_coordinates(self, inline_idx: int, xline_idx: int) -> Tuple[float, float]:
        """World (x, y) with the inline direction at ``inline_azimuth`` from north."""
        az = np.radians(self.inline_azimuth)
        di, dx = inline_idx * self.d_inline, xline_idx * self.d_xline
        return (self.x_origin + di * np.sin(az) + dx * np.cos(az),
                self.y_origin + di * np.cos(az) - dx * np.sin(az))

    def to_dict(self) -> Dict[str, Any]:
        return {k: getattr(self, k) for k in self.__dataclass_fields__}

    @classmethod
    def from_dict(cls, d: Dict[str, Any]) -> "OutputGrid":
        return cls(**d)


@dataclass
class MigrationConfig:
    """Kirchhoff PSTM configuration (aperture, angle, offsets, taper, weights,
    anti-alias, interpolation, fold handling)."""
    output_grid: OutputGrid = field(default_factory=OutputGrid)
    max_aperture_m: float = 5000.0
    max_angle_deg: float = 60.0
    max_offset_m: float = 10000.0
    min_offset_m: float = 0.0
    taper_width: float = 0.1
    traveltime_mode: TraveltimeMode = TraveltimeMode.STRAIGHT_RAY
    use_anisotropy: bool = False
    anisotropy_method: AnisotropyMethod = AnisotropyMethod.ANELLIPTIC
    weight_mode: WeightMode = WeightMode.SPREADING
    preserve_amplitudes: bool = False
    antialias_enabled: bool = True
    antialias_fmax: float = 80.0
    interpolation_mode: InterpolationMode = InterpolationMode.SINC
    min_fold: int = 1
    normalize_by_fold: bool = True
    metadata: Dict[str, Any] = field(default_factory=dict)

    def __post_init__(self):
        if self.max_aperture_m <= 0:
            raise ValueError(f"max_aperture_m must be positive, got {self.max_aperture_m}")
        if not 0 < self.max_angle_deg <= 90:
            raise ValueError(f"max_angle_deg must be in (0, 90], got {self.max_angle_deg}")
        if self.max_offset_m <= 0:
            raise ValueError(f"max_offset_m must be positive, got {self.max_offset_m}")
        if self.min_offset_m < 0:
            raise ValueError(f"min_offset_m must be non-negative, got {self.min_offset_m}")
        if self.min_offset_m >= self.max_offset_m:
            raise ValueError(f"min_offset_m ({self.min_offset_m}) must be less than "
                             f"max_offset_m ({self.max_offset_m})")
        if not 0 <= self.taper_width <= 1:
            raise ValueError(f"taper_width must be in [0, 1], got {self.taper_width}")
        if self.min_fold < 1:
            raise ValueError(f"min_fold must be >= 1, got {self.min_fold}")
        if self.antialias_fmax <= 0:
            raise ValueError(f"antialias_fmax must be positive, got {self.antialias_fmax}")

    @property
    def max_angle_rad(self) -> float:
        return float(np.radians(self.max_angle_deg))

    def to_dict(self) -> Dict[str, Any]:
        d = {k: getattr(self, k) for k in self.__dataclass_fields__}
        d["output_grid"] = self.output_grid.to_dict()
        for k in ("traveltime_mode", "anisotropy_method", "weight_mode", "interpolation_mode"):
            d[k] = d[k].value
        d["metadata"] = dict(self.metadata)
        return d

    @classmethod
    def from_dict(cls, d: Dict[str, Any]) -> "MigrationConfig":
        d = dict(d)
        grid = OutputGrid.from_dict(d.pop("output_grid"))
        return cls(output_grid=grid,
                   traveltime_mode=TraveltimeMode(d.pop("traveltime_mode", "straight_ray")),
                   weight_mode=WeightMode(d.pop("weight_mode", "spreading")),
                   interpolation_mode=InterpolationMode(d.pop("interpolation_mode", "sinc")),
                   anisotropy_method=AnisotropyMethod(d.pop("anisotropy_method", "anelliptic")),
                   **d)

    def copy(self) -> "MigrationConfig":
        return MigrationConfig.from_dict(self.to_dict())


# ---------------------------------------------------------------- geometry --
@dataclass
class MigrationGeometry:
    """Source/receiver coordinates per trace.  The reference stores them as
    float32; ``keep_float64=True`` keeps float64 world coordinates (UTM) so the
    grid origin can be subtracted before rounding."""
    source_x: np.ndarray
    source_y: np.ndarray
    receiver_x: np.ndarray
    receiver_y: np.ndarray
    source_z: Optional[np.ndarray] = None
    receiver_z: Optional[np.ndarray] = None
    trace_indices: Optional[np.ndarray] = None
    metadata: Dict[str, Any] = field(default_factory=dict)
    keep_float64: bool = False

    def __post_init__(self):
        dt = np.float64 if self.keep_float64 else np.float32
        self.source_x = np.asarray(self.source_x, dtype=dt)
        self.source_y = np.asarray(self.source_y, dtype=dt)
        self.receiver_x = np.asarray(self.receiver_x, dtype=dt)
        self.receiver_y = np.asarray(self.receiver_y, dtype=dt)
        n = len(self.source_x)
        for nm in ("source_y", "receiver_x", "receiver_y"):
            if len(getattr(self, nm)) != n:
                raise ValueError(f"{nm} length {len(getattr(self, nm))} != source_x length {n}")
        if self.trace_indices is not None:
            self.trace_indices = np.asarray(self.trace_indices, dtype=np.int32)

    @property
    def n_traces(self) -> int:
        return len(self.source_x)

    @property
    def offset(self) -> np.ndarray:
        return np.hypot(self.receiver_x - self.source_x,
                        self.receiver_y - self.source_y).astype(np.float32)

    @property
    def azimuth(self) -> np.ndarray:
        """Source-to-receiver azimuth in degrees [0, 360), clockwise from north."""
        az = np.degrees(np.arctan2(self.receiver_x - self.source_x,
                                   self.receiver_y - self.source_y))
        return ((az + 360.0) % 360.0).astype(np.float32)

    @property
    def cdp_x(self) -> np.ndarray:
        return ((self.source_x + self.receiver_x) / 2).astype(self.source_x.dtype)

    @property
    def cdp_y(self) -> np.ndarray:
        return ((self.source_y + self.receiver_y) / 2).astype(self.source_y.dtype)

    def filter_by_offset(self, min_offset: float, max_offset: float) -> "MigrationGeometry":
        off = self.offset
        return self._apply_mask((off >= min_offset) & (off <= max_offset))

    def filter_by_azimuth(self, min_azimuth: float, max_azimuth: float) -> "MigrationGeometry":
        return self._apply_mask(_azimuth_mask(self.azimuth, min_azimuth, max_azimuth))

    def filter_by_offset_azimuth(self, min_offset, max_offset, min_azimuth,
                                 max_azimuth) -> "MigrationGeometry":
        off = self.offset
        m = (off >= min_offset) & (off <= max_offset) & \
            _azimuth_mask(self.azimuth, min_azimuth, max_azimuth)
        return self._apply_mask(m)

    def get_indices_for_bin(self, min_offset, max_offset, min_azimuth=0.0,
                            max_azimuth=360.0) -> np.ndarray:
        off = self.offset
        m = (off >= min_offset) & (off <= max_offset) & \
            _azimuth_mask(self.azimuth, min_azimuth, max_azimuth)
        return np.nonzero(m)[0]

    def _apply_mask(self, m: np.ndarray) -> "MigrationGeometry":
        sel = lambda a: a[m] if a is not None else None
        return MigrationGeometry(self.source_x[m], self.source_y[m], self.receiver_x[m],
                                 self.receiver_y[m], sel(self.source_z), sel(self.receiver_z),
                                 sel(self.trace_indices), dict(self.metadata),
                                 keep_float64=self.keep_float64)


def _azimuth_mask(az: np.ndarray, lo: float, hi: float) -> np.ndarray:
    if lo <= hi:
        return (az >= lo) & (az <= hi)
    return (az >= lo) | (az <= hi)


@dataclass
class SeismicData:
    """Traces (n_samples, n_traces) with a sample rate in milliseconds."""
    traces: np.ndarray
    sample_rate: float
    headers: Optional[Dict[str, np.ndarray]] = None
    metadata: Dict[str, Any] = field(default_factory=dict)

    def __post_init__(self):
        if self.traces.ndim != 2:
            raise ValueError(f"Traces must be 2D array, got shape {self.traces.shape}")
        if self.sample_rate <= 0:
            raise ValueError(f"Sample rate must be positive, got {self.sample_rate}")
        if not np.issubdtype(self.traces.dtype, np.floating):
            self.traces = self.traces.astype(np.float32)

    @property
    def n_samples(self) -> int:
        return self.traces.shape[0]

    @property
    def n_traces(self) -> int:
        return self.traces.shape[1]

    @property
    def duration(self) -> float:
        return (self.n_samples - 1) * self.sample_rate

    @property
    def nyquist_freq(self) -> float:
        return 1000.0 / (2.0 * self.sample_rate)

    def get_time_axis(self) -> np.ndarray:
        return np.arange(self.n_samples) * self.sample_rate
