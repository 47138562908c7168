"""Velocity files -> ``VelocityModel``, and V_rms on the output grid on the device.

The readers and writers keep the names, arguments, unit handling and results
of the reference's utils/velocity_io.py (format detection :93-163, previews
:166-512, text :515-693, JSON :696-742, NumPy :745-836, auto :839-899,
conversion :902-1004, CDP-TV :1007-1093, SEG-Y :1096-1172, preview -> model
:1175-1288, per-CDP extraction :1291-1330):

* ASCII T-V pairs -> v(t) (``VelocityType.V_OF_Z``);
* ASCII CDP-T-V triplets -> v(t, cdp) (``V_OF_XZ``; every CDP resampled with
  ``np.interp`` onto the first CDP's sorted times);
* ASCII IL-XL-T-V -> v(t, inline) as the reference builds it, or, with
  ``read_velocity_ilxltv_3d``, the full v(t, inline, xline) cube (new);
* SEG-Y velocity traces -> v(t) or v(t, cdp).  segyio is not available here,
  so ``read_segy_traces`` reads the subset of SEG-Y rev 1 a velocity file
  uses (binary-header interval / sample count / format, trace headers CDP,
  inline, crossline, delay; IBM or IEEE float, 8/16/32-bit integers) and
  gives the sample times the way segyio does (first trace's delay plus
  i * interval);
* JSON / NPZ through ``VelocityModel.to_dict`` / ``from_dict``.

``velocity_grid`` is the device side: a laterally varying model is resampled
onto every (output time, output column) by one kernel (``pstm_velocity_grid``),
with the per-axis interval and fraction found on the host, in float64, with
the reference's linear extrapolation beyond the axis ends
(models/velocity_model.py:181-245).  The result stays in HBM as the
(n_times, n_columns) float32 V_rms array the migration kernels read.
"""
from __future__ import annotations

import ctypes as C
import json
import logging
import re
from dataclasses import dataclass, field
from enum import Enum
from pathlib import Path
from typing import Any, Dict, List, Optional, Tuple, Union

import numpy as np

from .models import (VelocityModel, VelocityType, _interp_axis, create_2d_velocity,
                     create_3d_velocity, interval_to_rms_velocity, rms_to_interval_velocity)

logger = logging.getLogger(__name__)

_SPLIT = re.compile(r"[,\s\t]+")
_TEXT_SUFFIXES = (".txt", ".vel", ".asc", ".dat", ".csv")


# ----------------------------------------------------------- units / lines --
def _seconds(t: np.ndarray, unit: str) -> np.ndarray:
    if unit == "ms":
        return t / 1000.0
    if unit == "us":
        return t / 1000000.0
    return t


def _metres_per_second(v: np.ndarray, unit: str) -> np.ndarray:
    if unit == "km/s":
        return v * 1000.0
    if unit == "ft/s":
        return v * 0.3048
    if unit == "ft/ms":
        return v * 304.8
    return v


def _data_lines(path: Path):
    """Non-empty lines that are not comments (# or //), stripped."""
    with open(path, "r") as f:
        for line in f:
            line = line.strip()
            if line and not line.startswith("#") and not line.startswith("//"):
                yield line


def _numeric_fields(parts: List[str]) -> int:
    n = 0
    for p in parts:
        try:
            float(p)
            n += 1
        except ValueError:
            pass
    return n


# -------------------------------------------------------- detection/preview --
class VelocityFileFormat(Enum):
    ASCII_TV = "ascii_tv"
    ASCII_CDPTV = "ascii_cdp_tv"
    ASCII_ILXLTV = "ascii_ilxl_tv"
    SEGY = "segy"
    JSON = "json"
    NPZ = "npz"
    UNKNOWN = "unknown"


@dataclass
class VelocityFileInfo:
    """What a preview learns about a velocity file (reference fields)."""
    path: Path
    format: VelocityFileFormat = VelocityFileFormat.UNKNOWN
    n_locations: int = 0
    n_time_samples: int = 0
    time_range: Tuple[float, float] = (0.0, 0.0)
    velocity_range: Tuple[float, float] = (0.0, 0.0)
    cdp_range: Optional[Tuple[int, int]] = None
    inline_range: Optional[Tuple[int, int]] = None
    xline_range: Optional[Tuple[int, int]] = None
    sample_interval: Optional[float] = None
    is_valid: bool = False
    error_message: Optional[str] = None
    raw_data: Optional[Dict[str, Any]] = field(default=None, repr=False)


def detect_velocity_format(filepath: Union[str, Path]) -> VelocityFileFormat:
    """By extension (.sgy/.segy, .json, .npy/.npz), else by the most common
    count of numeric fields on the first 20 data lines: 2 -> T-V, 3 -> CDP-T-V,
    4 or more -> IL-XL-T-V."""
    path = Path(filepath)
    if not path.exists():
        return VelocityFileFormat.UNKNOWN
    suffix = path.suffix.lower()
    if suffix in (".sgy", ".segy"):
        return VelocityFileFormat.SEGY
    if suffix == ".json":
        return VelocityFileFormat.JSON
    if suffix in (".npy", ".npz"):
        return VelocityFileFormat.NPZ
    try:
        counts = []
        for i, line in enumerate(_data_lines(path)):
            if i >= 20:
                break
            n = _numeric_fields(_SPLIT.split(line))
            if n:
                counts.append(n)
    except (OSError, UnicodeDecodeError) as e:
        logger.warning("Error detecting format: %s", e)
        return VelocityFileFormat.UNKNOWN
    if not counts:
        return VelocityFileFormat.UNKNOWN
    common = max(set(counts), key=counts.count)
    if common == 2:
        return VelocityFileFormat.ASCII_TV
    if common == 3:
        return VelocityFileFormat.ASCII_CDPTV
    if common >= 4:
        return VelocityFileFormat.ASCII_ILXLTV
    return VelocityFileFormat.UNKNOWN


def _columns(path: Path, n: int, int_cols: int):
    """Rows with at least n fields whose first n parse; the first int_cols
    fields are read as int(float(.))."""
    cols = [[] for _ in range(n)]
    for line in _data_lines(path):
        parts = _SPLIT.split(line)
        if len(parts) < n:
            continue
        try:
            vals = [int(float(p)) if j < int_cols else float(p) for j, p in enumerate(parts[:n])]
        except ValueError:
            continue
        for c, v in zip(cols, vals):
            c.append(v)
    return [np.array(c) for c in cols]


def _preview_tv(path: Path, info: VelocityFileInfo) -> VelocityFileInfo:
    t, v = _columns(path, 2, 0)
    if t.size == 0:
        info.error_message = "No valid data found"
        return info
    info.n_locations, info.n_time_samples = 1, int(t.size)
    info.time_range = (float(t.min()), float(t.max()))
    info.velocity_range = (float(v.min()), float(v.max()))
    if t.size > 1:
        d = np.diff(t)
        if np.allclose(d, d[0], rtol=0.01):
            info.sample_interval = float(d[0])
    info.raw_data = {"times": t, "velocities": v, "format": "tv"}
    info.is_valid = True
    return info


def _preview_cdptv(path: Path, info: VelocityFileInfo) -> VelocityFileInfo:
    cdp, t, v = _columns(path, 3, 1)
    if t.size == 0:
        info.error_message = "No valid data found"
        return info
    ucdp = np.unique(cdp)
    info.n_locations = int(ucdp.size)
    info.n_time_samples = int(t.size // ucdp.size)
    info.time_range = (float(t.min()), float(t.max()))
    info.velocity_range = (float(v.min()), float(v.max()))
    info.cdp_range = (int(ucdp.min()), int(ucdp.max()))
    info.raw_data = {"cdps": cdp, "times": t, "velocities": v, "unique_cdps": ucdp,
                     "format": "cdp_tv"}
    info.is_valid = True
    return info


def _preview_ilxltv(path: Path, info: VelocityFileInfo) -> VelocityFileInfo:
    il, xl, t, v = _columns(path, 4, 2)
    if t.size == 0:
        info.error_message = "No valid data found"
        return info
    uil, uxl = np.unique(il), np.unique(xl)
    # The reference counts np.unique over the flattened (inline, crossline)
    # pairs, i.e. the distinct numbers among both columns; kept as it is.
    n_loc = int(np.unique(np.stack([il, xl], 1)).size)
    info.n_locations = n_loc
    info.n_time_samples = int(t.size // n_loc)
    info.time_range = (float(t.min()), float(t.max()))
    info.velocity_range = (float(v.min()), float(v.max()))
    info.inline_range = (int(uil.min()), int(uil.max()))
    info.xline_range = (int(uxl.min()), int(uxl.max()))
    info.raw_data = {"inlines": il, "xlines": xl, "times": t, "velocities": v,
                     "unique_inlines": uil, "unique_xlines": uxl, "format": "ilxl_tv"}
    info.is_valid = True
    return info


def _preview_segy(path: Path, info: VelocityFileInfo, inline_byte: Optional[int],
                  xline_byte: Optional[int]) -> VelocityFileInfo:
    s = read_segy_traces(path, inline_byte or 189, xline_byte or 193)
    n_tr, n_s = s["traces"].shape
    head = s["traces"][:min(10, n_tr)]
    info.n_locations, info.n_time_samples = n_tr, n_s
    t = s["samples_ms"] / 1000.0
    info.time_range = (float(t.min()), float(t.max())) if n_s else (0.0, 0.0)
    info.velocity_range = (float(head.min()), float(head.max())) if head.size else (0.0, 0.0)
    info.sample_interval = s["interval_us"] / 1e6
    for key, attr in (("cdp", "cdp_range"), ("inline", "inline_range"),
                      ("xline", "xline_range")):
        a = s[key]
        if np.any(a != 0):
            setattr(info, attr, (int(a.min()), int(a.max())))
    info.raw_data = {"format": "segy", "filepath": str(path), "inline_byte": inline_byte,
                     "xline_byte": xline_byte}
    info.is_valid = True
    return info


def _preview_json(path: Path, info: VelocityFileInfo) -> VelocityFileInfo:
    with open(path, "r") as f:
        d = json.load(f)
    data = d.get("data")
    if isinstance(data, (int, float)):
        info.n_locations = info.n_time_samples = 1
        info.velocity_range = (float(data), float(data))
    elif isinstance(data, list):
        a = np.array(data)
        info.n_time_samples = int(a.shape[0])
        info.n_locations = int(a.shape[1]) if a.ndim > 1 else 1
        info.velocity_range = (float(a.min()), float(a.max()))
    if "z_axis" in d:
        z = np.array(d["z_axis"])
        info.time_range = (float(z.min()), float(z.max()))
        if z.size > 1:
            info.sample_interval = float(z[1] - z[0])
    info.raw_data = {"format": "json", "data": d}
    info.is_valid = True
    return info


def _preview_npz(path: Path, info: VelocityFileInfo) -> VelocityFileInfo:
    z = np.load(path, allow_pickle=True)
    a = z["data"]
    if a.ndim == 0:
        info.n_locations = info.n_time_samples = 1
        info.velocity_range = (float(a), float(a))
    else:
        info.n_time_samples = int(a.shape[0])
        info.n_locations = int(a.shape[1]) if a.ndim > 1 else 1
        info.velocity_range = (float(a.min()), float(a.max()))
    if "z_axis" in z and z["z_axis"].ndim > 0:
        ax = z["z_axis"]
        info.time_range = (float(ax.min()), float(ax.max()))
        if ax.size > 1:
            info.sample_interval = float(ax[1] - ax[0])
    info.raw_data = {"format": "npz", "filepath": str(path)}
    info.is_valid = True
    return info


def preview_velocity_file(filepath: Union[str, Path], inline_byte: Optional[int] = None,
                          xline_byte: Optional[int] = None) -> VelocityFileInfo:
    """Detect the format and parse the file; failures are reported in
    ``error_message`` with ``is_valid`` False (nothing is raised)."""
    path = Path(filepath)
    info = VelocityFileInfo(path=path)
    if not path.exists():
        info.error_message = f"File not found: {path}"
        return info
    info.format = detect_velocity_format(path)
    try:
        if info.format == VelocityFileFormat.SEGY:
            info = _preview_segy(path, info, inline_byte, xline_byte)
        elif info.format == VelocityFileFormat.JSON:
            info = _preview_json(path, info)
        elif info.format == VelocityFileFormat.NPZ:
            info = _preview_npz(path, info)
        elif info.format == VelocityFileFormat.ASCII_TV:
            info = _preview_tv(path, info)
        elif info.format == VelocityFileFormat.ASCII_CDPTV:
            info = _preview_cdptv(path, info)
        elif info.format == VelocityFileFormat.ASCII_ILXLTV:
            info = _preview_ilxltv(path, info)
        else:
            info.error_message = "Unknown file format"
    except Exception as e:  # reported, as the reference's preview does
        info.error_message = f"Preview error: {e}"
    return info


# ------------------------------------------------------------------ readers --
def read_velocity_text(filepath: str, velocity_type: str = "rms", time_column: int = 0,
                       velocity_column: int = 1, time_unit: str = "ms",
                       velocity_unit: str = "m/s", delimiter: Optional[str] = None,
                       skip_header: int = 0) -> VelocityModel:
    """T-V columns -> v(t), sorted by time (float32, seconds, m/s)."""
    path = Path(filepath)
    if not path.exists():
        raise FileNotFoundError(f"Velocity file not found: {path}")
    t, v = [], []
    with open(path, "r") as f:
        for i, line in enumerate(f):
            if i < skip_header:
                continue
            line = line.strip()
            if not line or line.startswith("#") or line.startswith("//"):
                continue
            parts = line.split(delimiter) if delimiter else line.split()
            if len(parts) <= max(time_column, velocity_column):
                continue
            try:
                tt, vv = float(parts[time_column]), float(parts[velocity_column])
            except ValueError:
                continue
            t.append(tt)
            v.append(vv)
    if not t:
        raise ValueError(f"No valid velocity data found in {path}")
    t = _seconds(np.array(t, np.float32), time_unit)
    v = _metres_per_second(np.array(v, np.float32), velocity_unit)
    order = np.argsort(t)
    return VelocityModel(data=v[order], z_axis=t[order], is_time=True,
                         metadata={"source_file": str(path), "velocity_type": velocity_type,
                                   "original_time_unit": time_unit,
                                   "original_velocity_unit": velocity_unit})


def _resample_locations(keys: np.ndarray, ukeys: np.ndarray, t: np.ndarray,
                        v: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Every location's v(t) resampled (np.interp, clamped at the ends) onto
    the first location's sorted times: (n_time, n_loc) float32, time axis."""
    axis = np.sort(t[keys == ukeys[0]])
    out = np.zeros((axis.size, ukeys.size), np.float32)
    for i, k in enumerate(ukeys):
        sel = keys == k
        tk, vk = t[sel], v[sel]
        order = np.argsort(tk)
        out[:, i] = np.interp(axis, tk[order], vk[order])
    return out, axis


def read_velocity_cdptv(filepath: Union[str, Path], time_unit: str = "ms",
                        velocity_unit: str = "m/s", velocity_type: str = "rms") -> VelocityModel:
    """CDP-T-V triplets -> v(t, cdp) (``V_OF_XZ``, x axis = CDP number)."""
    path = Path(filepath)
    if not path.exists():
        raise FileNotFoundError(f"Velocity file not found: {path}")
    info = preview_velocity_file(path)
    if not info.is_valid:
        raise ValueError(f"Failed to read velocity file: {info.error_message}")
    if info.format != VelocityFileFormat.ASCII_CDPTV:
        raise ValueError(f"Expected CDP-TV format, got {info.format.value}")
    r = info.raw_data
    t = _seconds(r["times"], time_unit)
    v = _metres_per_second(r["velocities"], velocity_unit)
    ucdp = r["unique_cdps"]
    vel, axis = _resample_locations(r["cdps"], ucdp, t, v)
    return create_2d_velocity(
        data=vel, z_axis=axis.astype(np.float32), x_axis=ucdp.astype(np.float32), is_time=True,
        metadata={"source_file": str(path), "velocity_type": velocity_type,
                  "cdp_range": (int(ucdp.min()), int(ucdp.max())),
                  "original_time_unit": time_unit, "original_velocity_unit": velocity_unit})


def read_velocity_ilxltv_3d(filepath: Union[str, Path], time_unit: str = "ms",
                            velocity_unit: str = "m/s",
                            velocity_type: str = "rms") -> VelocityModel:
    """IL-XL-T-V rows -> the full v(t, inline, xline) cube (``V_OF_XYZ``, x axis
    = inline number, y axis = crossline number).  Every (inline, crossline)
    location of the rectangle must be present; each is resampled onto the
    first location's sorted times as the 2-D readers do.  (The reference's
    IL-XL-T-V path keeps only the inline axis: ``velocity_info_to_model``.)"""
    path = Path(filepath)
    info = preview_velocity_file(path)
    if not info.is_valid:
        raise ValueError(f"Failed to read velocity file: {info.error_message}")
    if info.format != VelocityFileFormat.ASCII_ILXLTV:
        raise ValueError(f"Expected IL-XL-T-V format, got {info.format.value}")
    r = info.raw_data
    il, xl = r["inlines"], r["xlines"]
    uil, uxl = r["unique_inlines"], r["unique_xlines"]
    t = _seconds(r["times"], time_unit)
    v = _metres_per_second(r["velocities"], velocity_unit)
    # rows grouped by location (inline, crossline), times ascending in each
    order = np.lexsort((t, xl, il))
    il, xl, t, v = il[order], xl[order], t[order], v[order]
    new = np.ones(il.size, bool)
    new[1:] = (il[1:] != il[:-1]) | (xl[1:] != xl[:-1])
    starts = np.flatnonzero(new)
    if starts.size != uil.size * uxl.size:
        raise ValueError(f"IL-XL-T-V file covers {starts.size} of the {uil.size} x {uxl.size} "
                         "inline/crossline locations; a 3-D model needs all of them")
    ends = np.append(starts[1:], il.size)
    axis = t[starts[0]:ends[0]]  # the first location's (smallest inline, crossline) times
    cube = np.empty((axis.size, uil.size, uxl.size), np.float32)
    for g, (a, b) in enumerate(zip(starts, ends)):
        cube[:, g // uxl.size, g % uxl.size] = np.interp(axis, t[a:b], v[a:b])
    return create_3d_velocity(
        data=cube, z_axis=axis.astype(np.float32), x_axis=uil.astype(np.float32),
        y_axis=uxl.astype(np.float32), is_time=True,
        metadata={"source_file": str(path), "velocity_type": velocity_type,
                  "inline_range": info.inline_range, "xline_range": info.xline_range,
                  "lateral_axes": "inline_xline"})


def read_velocity_json(filepath: str) -> VelocityModel:
    path = Path(filepath)
    if not path.exists():
        raise FileNotFoundError(f"Velocity file not found: {path}")
    with open(path, "r") as f:
        m = VelocityModel.from_dict(json.load(f))
    m.metadata["source_file"] = str(path)
    return m


def write_velocity_json(model: VelocityModel, filepath: str, indent: int = 2) -> None:
    path = Path(filepath)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        json.dump(model.to_dict(), f, indent=indent)


def read_velocity_npy(filepath: str) -> VelocityModel:
    """.npz with 'data', optional 'z_axis'/'x_axis'/'y_axis', 'is_time' and a
    JSON 'metadata' string."""
    path = Path(filepath)
    if not path.exists():
        raise FileNotFoundError(f"Velocity file not found: {path}")
    z = np.load(path, allow_pickle=True)
    data = z["data"]
    data = float(data) if data.ndim == 0 else data
    ax = {k: z[k] if k in z else None for k in ("z_axis", "x_axis", "y_axis")}
    if ax["z_axis"] is not None and ax["z_axis"].ndim == 0:
        ax["z_axis"] = None
    meta = {}
    if "metadata" in z:
        try:
            meta = json.loads(str(z["metadata"]))
        except ValueError:
            meta = {}
    meta["source_file"] = str(path)
    is_time = bool(z["is_time"]) if "is_time" in z else True
    return VelocityModel(data=data, z_axis=ax["z_axis"], x_axis=ax["x_axis"],
                         y_axis=ax["y_axis"], is_time=is_time, metadata=meta)


def write_velocity_npy(model: VelocityModel, filepath: str) -> None:
    path = Path(filepath)
    if not path.suffix:
        path = path.with_suffix(".npz")
    path.parent.mkdir(parents=True, exist_ok=True)
    out = {"data": model.data if isinstance(model.data, np.ndarray) else np.array(model.data),
           "is_time": model.is_time, "metadata": json.dumps(model.metadata, default=str)}
    for k in ("z_axis", "x_axis", "y_axis"):
        if getattr(model, k) is not None:
            out[k] = getattr(model, k)
    np.savez(path, **out)


def write_velocity_text(model: VelocityModel, filepath: str, time_unit: str = "ms",
                        velocity_unit: str = "m/s", delimiter: str = "\t", header: bool = True,
                        precision: int = 2) -> None:
    """A constant model as two rows (t = 0 and 10000), a v(t) model row by row."""
    path = Path(filepath)
    path.parent.mkdir(parents=True, exist_ok=True)
    scale = {"ft/s": 1 / 0.3048, "km/s": 1 / 1000.0}.get(velocity_unit, 1.0)
    with open(path, "w") as f:
        if model.velocity_type == VelocityType.CONSTANT:
            if header:
                f.write("# Constant velocity model\n")
                f.write(f"# Time({time_unit}){delimiter}Velocity({velocity_unit})\n")
            v = model.data * scale
            f.write(f"0.0{delimiter}{v:.{precision}f}\n")
            f.write(f"10000.0{delimiter}{v:.{precision}f}\n")
            return
        t = np.asarray(model.z_axis) * (1000.0 if time_unit == "ms" else 1.0)
        v = np.asarray(model.data) * scale
        if header:
            f.write(f"# Velocity model: {model.velocity_type.value}\n")
            f.write(f"# v0={model.v0:.0f} m/s, gradient={model.gradient:.4f}\n")
            f.write(f"# Time({time_unit}){delimiter}Velocity({velocity_unit})\n")
        for tt, vv in zip(t, v):
            f.write(f"{tt:.{precision}f}{delimiter}{vv:.{precision}f}\n")


def read_velocity_auto(filepath: str, **kwargs) -> VelocityModel:
    """By extension: text (.txt .vel .asc .dat .csv, and any other), JSON, NPZ."""
    path = Path(filepath)
    s = path.suffix.lower()
    if s == ".json":
        return read_velocity_json(path)
    if s in (".npy", ".npz"):
        return read_velocity_npy(path)
    if s not in _TEXT_SUFFIXES:
        logger.warning("Unknown extension %s, trying text format", s)
    return read_velocity_text(path, **kwargs)


def write_velocity_auto(model: VelocityModel, filepath: str, **kwargs) -> None:
    path = Path(filepath)
    s = path.suffix.lower()
    if s in _TEXT_SUFFIXES:
        write_velocity_text(model, path, **kwargs)
    elif s in (".npy", ".npz"):
        write_velocity_npy(model, path)
    else:
        if s != ".json":
            logger.warning("Unknown extension %s, using JSON format", s)
        write_velocity_json(model, path, **kwargs)


def convert_velocity_file(input_path: str, output_path: str, input_type: str = "rms",
                          output_type: str = "interval", **read_kwargs) -> VelocityModel:
    """Read a v(t) file, convert RMS <-> interval (Dix), write it."""
    m = read_velocity_auto(input_path, velocity_type=input_type, **read_kwargs)
    if m.velocity_type != VelocityType.V_OF_Z:
        raise ValueError("Velocity conversion only supported for 1D v(z) models")
    if input_type != output_type:
        conv = {("rms", "interval"): rms_to_interval_velocity,
                ("interval", "rms"): interval_to_rms_velocity}.get((input_type, output_type))
        if conv is not None:
            t, v = conv(m.z_axis, m.data)
            m = VelocityModel(data=v, z_axis=t, is_time=m.is_time,
                              metadata={**m.metadata, "velocity_type": output_type})
    write_velocity_auto(m, output_path)
    return m


def create_velocity_from_picks(picks: List[Tuple[float, float]], dt: float = 0.004,
                               t_max: Optional[float] = None,
                               velocity_type: str = "rms") -> VelocityModel:
    """(time s, velocity) picks -> v(t) on a regular axis 0, dt, ... t_max."""
    if not picks:
        raise ValueError("No velocity picks provided")
    picks = sorted(picks, key=lambda p: p[0])
    tp = np.array([p[0] for p in picks], np.float32)
    vp = np.array([p[1] for p in picks], np.float32)
    t_max = tp[-1] if t_max is None else t_max
    axis = np.arange(0, t_max + dt, dt, dtype=np.float32)
    return VelocityModel(data=np.interp(axis, tp, vp).astype(np.float32), z_axis=axis,
                         is_time=True, metadata={"velocity_type": velocity_type,
                                                 "source": "picks", "n_picks": len(picks)})


# -------------------------------------------------------------------- SEG-Y --
_SEGY_SAMPLE = {1: (4, "ibm"), 2: (4, ">i4"), 3: (2, ">i2"), 5: (4, ">f4"), 8: (1, "i1")}


def _be(buf: np.ndarray, offset: int, nbytes: int) -> int:
    return int.from_bytes(bytes(buf[offset:offset + nbytes]), "big", signed=True)


def ibm_to_ieee(words: np.ndarray) -> np.ndarray:
    """IBM System/360 single precision (sign, 7-bit base-16 exponent excess 64,
    24-bit fraction) -> float32."""
    w = np.asarray(words, np.uint32)
    sign = np.where(w >> 31, -1.0, 1.0)
    expo = ((w >> 24) & 0x7F).astype(np.int64) - 64
    frac = (w & 0x00FFFFFF).astype(np.float64) / float(1 << 24)
    return (sign * frac * np.power(16.0, expo)).astype(np.float32)


def ieee_to_ibm(x: np.ndarray) -> np.ndarray:
    """float -> IBM single precision words (fraction rounded to nearest)."""
    x = np.asarray(x, np.float64)
    out = np.zeros(x.shape, np.uint32)
    nz = x != 0
    a = np.abs(x[nz])
    e = np.floor(np.log2(a) / 4.0).astype(np.int64) + 1  # 16^(e-1) <= a < 16^e
    frac = a / np.power(16.0, e)
    lo = frac < 1.0 / 16
    e[lo] -= 1
    frac[lo] *= 16
    hi = frac >= 1.0
    e[hi] += 1
    frac[hi] /= 16
    m = np.rint(frac * (1 << 24)).astype(np.int64)
    carry = m >= (1 << 24)
    m[carry] >>= 4
    e[carry] += 1
    word = (np.where(x[nz] < 0, 1, 0).astype(np.uint64) << 31) | \
        (np.clip(e + 64, 0, 127).astype(np.uint64) << 24) | m.astype(np.uint64)
    out[nz] = word.astype(np.uint32)
    return out


def read_segy_traces(filepath: Union[str, Path], inline_byte: int = 189,
                     xline_byte: int = 193) -> Dict[str, Any]:
    """Traces and the headers a velocity file needs, from a SEG-Y file.

    Returns ``traces`` (n_traces, n_samples) float32, ``samples_ms`` (the
    first trace's delay recording time + i * interval, as segyio's
    ``f.samples``), ``interval_us`` and per-trace int32 ``cdp`` (bytes 21-24),
    ``inline`` and ``xline`` (at the given 1-based bytes).  The sample
    interval and count come from the binary header (bytes 3217 and 3221),
    else from the first trace header (bytes 117 and 115)."""
    raw = np.fromfile(str(filepath), np.uint8)
    if raw.size < 3600:
        raise ValueError(f"{filepath}: too short for a SEG-Y file")
    interval = _be(raw, 3216, 2) & 0xFFFF
    n_s = _be(raw, 3220, 2) & 0xFFFF
    fmt = _be(raw, 3224, 2)
    n_ext = max(_be(raw, 3504, 2), 0)
    start = 3600 + 3200 * n_ext
    if fmt not in _SEGY_SAMPLE:
        raise ValueError(f"{filepath}: unsupported SEG-Y sample format {fmt}")
    if raw.size >= start + 240:
        if n_s == 0:
            n_s = _be(raw, start + 114, 2) & 0xFFFF
        if interval == 0:
            interval = _be(raw, start + 116, 2) & 0xFFFF
    nbytes, kind = _SEGY_SAMPLE[fmt]
    rec = 240 + n_s * nbytes
    n_tr = (raw.size - start) // rec
    block = raw[start:start + n_tr * rec].reshape(n_tr, rec)
    hdr = np.ascontiguousarray(block[:, :240])

    def field32(byte1: int) -> np.ndarray:
        return hdr[:, byte1 - 1:byte1 + 3].copy().view(">i4").reshape(-1).astype(np.int32)

    body = np.ascontiguousarray(block[:, 240:])
    if kind == "ibm":
        data = ibm_to_ieee(body.view(">u4").reshape(n_tr, n_s))
    else:
        data = body.view(kind).reshape(n_tr, n_s).astype(np.float32)
    delay = _be(hdr[0], 108, 2) if n_tr else 0
    return {"traces": data, "samples_ms": delay + np.arange(n_s) * (interval / 1000.0),
            "interval_us": interval, "format": fmt, "cdp": field32(21),
            "inline": field32(inline_byte), "xline": field32(xline_byte)}


def write_segy_traces(filepath: Union[str, Path], traces: np.ndarray, interval_us: int,
                      cdp=None, inline=None, xline=None, fmt: int = 5,
                      delay_ms: int = 0) -> None:
    """A minimal SEG-Y rev 1 file: blank textual header, binary header
    (interval, sample count, format), one 240-byte header per trace (CDP,
    delay, sample count, interval, inline at 189, crossline at 193)."""
    tr = np.asarray(traces, np.float32)
    n_tr, n_s = tr.shape
    if fmt not in (1, 5):
        raise ValueError("write_segy_traces writes IBM (1) or IEEE (5) float samples")
    head = bytearray(b" " * 3200) + bytearray(400)
    head[3216:3218] = int(interval_us).to_bytes(2, "big")
    head[3220:3222] = int(n_s).to_bytes(2, "big")
    head[3224:3226] = int(fmt).to_bytes(2, "big")
    head[3500:3502] = (256).to_bytes(2, "big")  # SEG-Y revision 1.0
    zeros = np.zeros(n_tr, np.int64)
    cols = [np.asarray(a if a is not None else zeros, np.int64) for a in (cdp, inline, xline)]
    th = np.zeros((n_tr, 240), np.uint8)
    for byte1, vals in ((21, cols[0]), (189, cols[1]), (193, cols[2])):
        th[:, byte1 - 1:byte1 + 3] = vals.astype(">i4").view(np.uint8).reshape(n_tr, 4)
    th[:, 108:110] = np.full(n_tr, delay_ms, ">i2").view(np.uint8).reshape(n_tr, 2)
    th[:, 114:116] = np.full(n_tr, n_s, ">u2").view(np.uint8).reshape(n_tr, 2)
    th[:, 116:118] = np.full(n_tr, interval_us, ">u2").view(np.uint8).reshape(n_tr, 2)
    body = ieee_to_ibm(tr).astype(">u4") if fmt == 1 else tr.astype(">f4")
    rec = np.concatenate([th, body.view(np.uint8).reshape(n_tr, 4 * n_s)], axis=1)
    with open(filepath, "wb") as f:
        f.write(bytes(head))
        f.write(rec.tobytes())


def read_velocity_segy(filepath: Union[str, Path], velocity_type: str = "rms") -> VelocityModel:
    """One trace -> v(t); several -> v(t, cdp) with the CDP numbers as x axis
    (trace numbers 0.. when every CDP header is 0)."""
    path = Path(filepath)
    if not path.exists():
        raise FileNotFoundError(f"Velocity file not found: {path}")
    s = read_segy_traces(path)
    t = (s["samples_ms"] / 1000.0).astype(np.float32)
    tr = s["traces"]
    meta = {"source_file": str(path), "velocity_type": velocity_type, "format": "segy"}
    if tr.shape[0] == 1:
        return VelocityModel(data=tr[0].astype(np.float32), z_axis=t, is_time=True,
                             metadata=meta)
    cdp = s["cdp"]
    has = bool(np.any(cdp != 0))
    x = cdp.astype(np.float32) if has else np.arange(tr.shape[0], dtype=np.float32)
    meta["cdp_range"] = (int(cdp.min()), int(cdp.max())) if has else None
    return create_2d_velocity(data=np.ascontiguousarray(tr.T), z_axis=t, x_axis=x,
                              is_time=True, metadata=meta)


def velocity_info_to_model(info: VelocityFileInfo, velocity_type: str = "rms",
                           time_unit: str = "ms", velocity_unit: str = "m/s") -> VelocityModel:
    """A previewed file -> model; IL-XL-T-V keeps the inline axis only, as the
    reference does (``read_velocity_ilxltv_3d`` keeps both)."""
    if not info.is_valid:
        raise ValueError(f"Invalid velocity file: {info.error_message}")
    r = info.raw_data
    fmt = r.get("format", "")
    if fmt == "tv":
        t = _seconds(r["times"].copy(), time_unit)
        v = _metres_per_second(r["velocities"].copy(), velocity_unit)
        return VelocityModel(data=v.astype(np.float32), z_axis=t.astype(np.float32),
                             is_time=True, metadata={"source_file": str(info.path),
                                                     "velocity_type": velocity_type})
    if fmt == "cdp_tv":
        return read_velocity_cdptv(info.path, time_unit=time_unit, velocity_unit=velocity_unit,
                                   velocity_type=velocity_type)
    if fmt == "ilxl_tv":
        t = _seconds(r["times"].copy(), time_unit)
        v = _metres_per_second(r["velocities"].copy(), velocity_unit)
        uil = r["unique_inlines"]
        vel, axis = _resample_locations(r["inlines"], uil, t, v)
        return create_2d_velocity(
            data=vel, z_axis=axis.astype(np.float32), x_axis=uil.astype(np.float32),
            is_time=True, metadata={"source_file": str(info.path), "velocity_type": velocity_type,
                                    "inline_range": info.inline_range,
                                    "xline_range": info.xline_range})
    if fmt == "segy":
        return read_velocity_segy(info.path, velocity_type=velocity_type)
    if fmt == "json":
        return read_velocity_json(str(info.path))
    if fmt == "npz":
        return read_velocity_npy(str(info.path))
    raise ValueError(f"Unknown velocity format: {fmt}")


def get_velocity_at_cdp(model: VelocityModel, cdp: int,
                        times: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
    """(times, velocities) of one CDP: a 2-D model interpolated at x = cdp."""
    if model.velocity_type == VelocityType.CONSTANT:
        if times is None:
            times = np.array([0.0, 6.0], np.float32)
        return times, np.full_like(times, model.data)
    if model.velocity_type == VelocityType.V_OF_Z:
        if times is None:
            return model.z_axis, model.data
        return times, np.interp(times, model.z_axis, model.data).astype(np.float32)
    if model.velocity_type == VelocityType.V_OF_XZ:
        if times is None:
            times = model.z_axis
        return times, model.get_velocity_at(times, x=float(cdp))
    raise ValueError(f"Unsupported velocity type: {model.velocity_type}")


def get_velocity_summary(model: VelocityModel) -> str:
    lines = [f"Type: {model.velocity_type.value}",
             f"Domain: {'time' if model.is_time else 'depth'}"]
    if model.velocity_type == VelocityType.CONSTANT:
        lines.append(f"Velocity: {model.data:.0f} m/s")
    else:
        d = np.asarray(model.data)
        lines.append(f"Velocity range: {d.min():.0f} - {d.max():.0f} m/s")
        z = np.asarray(model.z_axis)
        unit = "s" if model.is_time else "m"
        lines.append(f"{'Time' if model.is_time else 'Depth'} range: "
                     f"{z.min():.3f} - {z.max():.3f} {unit} ({z.size} samples)")
        if model.x_axis is not None:
            lines.append(f"Lateral x: {np.min(model.x_axis):.0f} - {np.max(model.x_axis):.0f} "
                         f"({len(model.x_axis)} locations)")
        if model.y_axis is not None:
            lines.append(f"Lateral y: {np.min(model.y_axis):.0f} - {np.max(model.y_axis):.0f} "
                         f"({len(model.y_axis)} locations)")
    return "\n".join(lines)


# ---------------------------------------------------------- device V_rms grid --
def axis_tables(model: VelocityModel, t_s: np.ndarray, col_x: np.ndarray,
                col_y: Optional[np.ndarray] = None):
    """Per-axis (interval index int32, fraction float64) for the output times
    and columns: the host half of ``velocity_grid``."""
    if model.velocity_type not in (VelocityType.V_OF_XZ, VelocityType.V_OF_XYZ):
        raise ValueError("axis tables are for laterally varying (2-D / 3-D) models")
    iz, wz = _interp_axis(model.z_axis, np.asarray(t_s, np.float64))
    ix, wx = _interp_axis(model.x_axis, np.asarray(col_x, np.float64))
    tabs = [iz.astype(np.int32), wz.astype(np.float64), ix.astype(np.int32),
            wx.astype(np.float64)]
    if model.velocity_type == VelocityType.V_OF_XYZ:
        if col_y is None:
            raise ValueError("x, y coordinates required for 3D velocity model")
        iy, wy = _interp_axis(model.y_axis, np.asarray(col_y, np.float64))
        tabs += [iy.astype(np.int32), wy.astype(np.float64)]
    else:
        tabs += [None, None]
    return tabs


class VelocityGridder:
    """A laterally varying model and its per-axis tables resident on the
    device; ``run()`` launches the resampling kernel into ``out``, the
    (n_t, n_cols) float32 V_rms array."""

    def __init__(self, model: VelocityModel, t_s: np.ndarray, col_x: np.ndarray,
                 col_y: Optional[np.ndarray] = None, device=None):
        import torch
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise ValueError("velocity_grid runs on a CUDA device only")
        if not model.is_time:
            raise ValueError("PSTM needs a time-domain velocity model (is_time=True)")
        tabs = axis_tables(model, t_s, col_x, col_y)
        d = np.ascontiguousarray(model.data, np.float32)
        self.shape3 = (d.shape[0], d.shape[1], d.shape[2] if d.ndim == 3 else 1)
        self.n_t = int(np.asarray(t_s).shape[0])
        self.n_cols = int(np.asarray(col_x).shape[0])
        with torch.cuda.device(self.device):
            self.model = torch.from_numpy(d).to(self.device)
            self.tabs = [torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
                         if a is not None else None for a in tabs]
            self.out = torch.empty((self.n_t, self.n_cols), dtype=torch.float32,
                                   device=self.device)

    def run(self):
        import torch

        from . import _lib
        ptr = lambda x: C.c_void_p(x.data_ptr()) if x is not None else None
        t = self.tabs
        _lib.check(_lib.lib().pstm_velocity_grid(
            ptr(self.model), *self.shape3, ptr(t[0]), ptr(t[1]), self.n_t, ptr(t[2]), ptr(t[3]),
            ptr(t[4]), ptr(t[5]), self.n_cols, ptr(self.out),
            C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))
        return self.out


def velocity_grid(model: VelocityModel, t_s: np.ndarray, col_x: np.ndarray,
                  col_y: Optional[np.ndarray] = None, device=None):
    """V_rms at the output samples as a torch CUDA tensor: shape (1,) for a
    constant model, (n_t,) for v(t), (n_t, n_cols) for a 2-D / 3-D model.
    ``col_x`` / ``col_y`` are each output column's position in the model's
    lateral units (coordinates, or inline / crossline numbers for a model read
    by ``read_velocity_ilxltv_3d``)."""
    import torch
    dev = torch.device(device) if device is not None else torch.device("cuda")
    if dev.type != "cuda":
        raise ValueError("velocity_grid runs on a CUDA device only")
    if not model.is_time:
        raise ValueError("PSTM needs a time-domain velocity model (is_time=True)")
    t_s = np.asarray(t_s, np.float64)
    if model.velocity_type == VelocityType.CONSTANT:
        return torch.full((1,), float(model.data), dtype=torch.float32, device=dev)
    if model.velocity_type == VelocityType.V_OF_Z:
        v = np.interp(t_s, model.z_axis, model.data).astype(np.float32)
        return torch.from_numpy(v).to(dev)
    # the model and tables go back to the caching allocator on this stream,
    # after the kernel
    return VelocityGridder(model, t_s, col_x, col_y, dev).run()
