"""Engine-side velocity model: V_rms(t) for constant, linear-gradient and
tabulated v(z) interval velocities.

Same interface and formulas as processors/migration/velocity_model.py:30-345:
* constant: V_rms = v0                                               (:92-122)
* gradient v(z) = v0 + k z: z ~ v0 t_owt + k v0 t_owt^2 / 2,
  V_rms^2 = v0^2 + v0 k z + (k z)^2 / 3, V_rms = v0 for t < 1 ms      (:124-210)
* file: trapezoid one-way times and cumulative v^2 dt, interpolated  (:212-261)
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch


@dataclass
class VelocityModel:
    velocity_type: str
    v0: float
    gradient: float = 0.0
    velocity_array: Optional[np.ndarray] = None
    z_axis: Optional[np.ndarray] = None

    def __post_init__(self):
        if self.velocity_type not in ("constant", "gradient", "file"):
            raise ValueError(f"Unknown velocity type: {self.velocity_type}")
        if self.velocity_type == "file" and self.velocity_array is None:
            raise ValueError("velocity_array required for 'file' type")
        self._table = None

    def interval_velocity(self, z):
        if self.velocity_type == "constant":
            return np.full_like(np.asarray(z, np.float64), self.v0) if np.ndim(z) else self.v0
        if self.velocity_type == "gradient":
            return self.v0 + self.gradient * np.asarray(z)
        return np.interp(z, self.z_axis, self.velocity_array)

    def rms_velocity_at_time(self, t_ms):
        """V_rms at two-way time t (ms); numpy arrays in, float32 arrays out.
        A float32 torch tensor gives a float32 tensor on its device, with the
        gradient formula evaluated in float32 in the reference's order
        (velocity_model.py:155-175), as the reference's tensor branch does."""
        if isinstance(t_ms, torch.Tensor):
            return self._rms_velocity_tensor(t_ms)
        scalar = np.ndim(t_ms) == 0
        t = np.asarray(t_ms, np.float64)
        if self.velocity_type == "constant" or (self.velocity_type == "gradient"
                                                and abs(self.gradient) < 1e-10):
            out = np.full(t.shape, self.v0, np.float32)
        elif self.velocity_type == "gradient":
            v0, k = self.v0, self.gradient
            tw = t / 2000.0
            z = np.maximum(v0 * tw + 0.5 * k * v0 * tw * tw, 0.0)
            vs = v0 * v0 + v0 * k * z + (k * k * z * z) / 3.0
            out = np.where(t < 1.0, v0, np.sqrt(np.maximum(vs, v0 * v0 * 0.5))).astype(np.float32)
        else:
            if self._table is None:
                self._build_table()
            tt, vv = self._table
            out = np.interp(t, tt, vv).astype(np.float32)
        return float(out) if scalar else out

    def _rms_velocity_tensor(self, t: torch.Tensor) -> torch.Tensor:
        if self.velocity_type == "constant" or (self.velocity_type == "gradient"
                                                and abs(self.gradient) < 1e-10):
            return torch.full_like(t, self.v0)
        if self.velocity_type == "gradient":
            v0, k = self.v0, self.gradient
            # divisors as tensors: a CUDA tensor divided by a Python number is
            # multiplied by the float32 reciprocal, which rounds differently
            tw = t / torch.tensor(2000.0, dtype=t.dtype, device=t.device)
            z = torch.clamp(v0 * tw + 0.5 * k * v0 * tw * tw, min=0)
            vs = v0 * v0 + v0 * k * z + (k * k * z * z) / torch.tensor(3.0, dtype=t.dtype,
                                                                         device=t.device)
            v = torch.sqrt(torch.clamp(vs, min=v0 * v0 * 0.5))
            return torch.where(t < 1.0, torch.full_like(v, v0), v)
        out = self.rms_velocity_at_time(t.detach().cpu().numpy())
        return torch.from_numpy(np.asarray(out, np.float32)).to(t.device)

    def _build_table(self):
        z = np.asarray(self.z_axis, np.float64)
        v = np.asarray(self.velocity_array, np.float64)
        vavg = 0.5 * (v[:-1] + v[1:])
        dt = np.diff(z) / vavg
        t_owt = np.concatenate([[0.0], np.cumsum(dt)])
        v2 = np.concatenate([[0.0], np.cumsum(vavg ** 2 * dt)])
        with np.errstate(divide="ignore", invalid="ignore"):
            vs = v2 / np.maximum(t_owt, 1e-10)
        vs[0] = v[0] ** 2
        self._table = (t_owt * 2000.0, np.sqrt(vs).astype(np.float32))

    def get_summary(self) -> str:
        if self.velocity_type == "constant":
            return f"Constant velocity: {self.v0:.0f} m/s"
        if self.velocity_type == "gradient":
            return f"Linear gradient: v(z) = {self.v0:.0f} + {self.gradient:.4f}*z m/s"
        return f"From file: {len(self.velocity_array)} points, v0={self.velocity_array[0]:.0f} m/s"


def create_velocity_model(velocity_type: str, v0: float, gradient: float = 0.0,
                          velocity_file: Optional[str] = None) -> VelocityModel:
    if velocity_type == "constant":
        return VelocityModel("constant", v0)
    if velocity_type == "gradient":
        return VelocityModel("gradient", v0, gradient=gradient)
    if velocity_type == "file":
        if velocity_file is None:
            raise ValueError("velocity_file required for 'file' type")
        data = np.loadtxt(velocity_file)
        return VelocityModel("file", float(data[0, 1]), velocity_array=data[:, 1].astype(np.float32),
                             z_axis=data[:, 0].astype(np.float32))
    raise ValueError(f"Unknown velocity type: {velocity_type}")


def create_velocity_model_from_config(config: dict) -> VelocityModel:
    return create_velocity_model(config.get("velocity_type", "constant"),
                                 config.get("velocity_v0", 2500.0),
                                 config.get("velocity_gradient", 0.0),
                                 config.get("velocity_file", None))
