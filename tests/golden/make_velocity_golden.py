"""Golden vectors for velocity ingestion, made by running the reference itself.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_velocity_golden.py /path/to/reference

Writes ``velocity_io.npz``: the text of four velocity files (T-V, CDP-T-V with
irregular and unsorted picks, IL-XL-T-V, and one with comments, commas and a
header line), the format the reference detects for each, the models its
readers build (utils/velocity_io.py), and the reference ``VelocityModel``'s
2-D and 3-D interpolation (models/velocity_model.py:181-245) at points inside
and outside the model's axes.  The reference is imported through the same
namespace-package shim as ``make_golden.py``; nothing is written into its tree.
"""
from __future__ import annotations

import importlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import import_reference  # noqa: E402


def velocity_files(rs: np.random.RandomState):
    """Deterministic file texts."""
    tv = "\n".join(f"{t:.1f} {1480 + 0.9 * t + rs.uniform(-5, 5):.2f}"
                   for t in (0, 250, 600, 1000, 1700, 2500, 4000))
    rows = ["# CDP  TIME(ms)  VRMS", "// picked velocities"]
    for cdp in (1200, 1100, 1150, 1300):  # not in order
        times = np.sort(rs.uniform(0, 4000, 6).round(1))
        times[0] = 0.0
        for t in rs.permutation(times):  # picks not in time order either
            rows.append(f"{cdp}\t{t:.1f}\t{1500 + 0.8 * t + 0.5 * (cdp - 1100) + rs.uniform(-20, 20):.2f}")
    cdptv = "\n".join(rows)
    rows = []
    for il in (100, 102, 104):
        for xl in (10, 20, 30, 40):
            for t in (0.0, 800.0, 1600.0, 3200.0):
                rows.append(f"{il} {xl} {t:.1f} {1500 + 0.7 * t + 3 * (il - 100) + 0.5 * xl:.2f}")
    ilxltv = "\n".join(rows)
    mixed = "Time,Velocity\n# header above is not numeric\n0,1500\n500,1650.5\n1000,1900\n" \
            "2000,2300.25\n\n3000,2600\n"
    return {"tv": tv, "cdptv": cdptv, "ilxltv": ilxltv, "mixed": mixed}


def main(ref_root: str):
    _, _, _, vel, _, _ = import_reference(ref_root)
    vio = importlib.import_module("utils.velocity_io")
    rs = np.random.RandomState(2024)
    texts = velocity_files(rs)
    out = {f"text_{k}": np.array(v) for k, v in texts.items()}
    with tempfile.TemporaryDirectory() as d:
        paths = {}
        for k, v in texts.items():
            paths[k] = os.path.join(d, f"{k}.txt")
            with open(paths[k], "w") as f:
                f.write(v + "\n")
        for k, p in paths.items():
            out[f"format_{k}"] = np.array(vio.detect_velocity_format(p).value)
        m = vio.read_velocity_text(paths["tv"])
        out["tv_t"], out["tv_v"] = m.z_axis, m.data
        m = vio.read_velocity_text(paths["mixed"], delimiter=",", skip_header=1,
                                   time_unit="ms", velocity_unit="km/s")
        out["mixed_t"], out["mixed_v"] = m.z_axis, m.data
        m = vio.read_velocity_cdptv(paths["cdptv"])
        out["cdptv_t"], out["cdptv_x"], out["cdptv_v"] = m.z_axis, m.x_axis, m.data
        info = vio.preview_velocity_file(paths["cdptv"])
        out["cdptv_preview"] = np.array([info.n_locations, info.n_time_samples,
                                         info.cdp_range[0], info.cdp_range[1]], np.int64)
        info = vio.preview_velocity_file(paths["ilxltv"])
        m = vio.velocity_info_to_model(info)
        out["ilxl_t"], out["ilxl_x"], out["ilxl_v"] = m.z_axis, m.x_axis, m.data
        out["ilxl_preview"] = np.array([info.n_locations, info.n_time_samples,
                                        *info.inline_range, *info.xline_range], np.int64)
        t_q = np.array([0.0, 0.3, 1.234, 2.0, 3.9], np.float32)
        tq, vq = vio.get_velocity_at_cdp(vio.read_velocity_cdptv(paths["cdptv"]), 1175, t_q)
        out["cdp1175_v"] = np.asarray(vq)

    # 2-D and 3-D interpolation with extrapolation past every axis end
    z = np.array([0.0, 0.5, 1.2, 2.0, 3.5], np.float32)
    x = np.array([0.0, 400.0, 900.0, 1500.0], np.float32)
    y = np.array([-100.0, 300.0, 700.0], np.float32)
    cube = (1500 + 600 * z[:, None, None] + 0.2 * x[None, :, None] - 0.1 * y[None, None, :]
            + rs.uniform(-30, 30, (z.size, x.size, y.size))).astype(np.float32)
    m3 = vel.create_3d_velocity(cube, z, x, y, is_time=True)
    m2 = vel.create_2d_velocity(cube[:, :, 1], z, x, is_time=True)
    n = 400
    pz = rs.uniform(-0.3, 4.0, n).astype(np.float64)
    px = rs.uniform(-200.0, 1800.0, n).astype(np.float64)
    py = rs.uniform(-300.0, 900.0, n).astype(np.float64)
    pz[:5] = z[:5]  # on the nodes
    px[:4] = x
    out.update(m_z=z, m_x=x, m_y=y, m_cube=cube, p_z=pz, p_x=px, p_y=py,
               v3=np.asarray(m3.get_velocity_at(pz, px, py), np.float32),
               v2=np.asarray(m2.get_velocity_at(pz, px), np.float32))
    np.savez_compressed(os.path.join(HERE, "velocity_io.npz"), **out)
    print("wrote", os.path.join(HERE, "velocity_io.npz"), sorted(out))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SEISPROC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the SeisProc checkout> "
                 "(or set SEISPROC_REFERENCE)")
    main(ref)
