"""Golden vectors for the time-domain RMS operator, made by running the reference.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_time_domain_golden.py /path/to/reference

Writes ``time_domain_rms.npz``: four seeded surveys migrated by the reference's
``MigrationEngine.migrate_bin_time_domain_rms``
(processors/migration/migration_engine.py:633-802, kernel
kirchhoff_kernel.py:1313-1783) on the CPU:

* ``c0``: constant V, time-dependent aperture, azimuth 0, no normalisation;
* ``c1``: linear-gradient V, rotated grid (30 deg), t_min 40 ms, fixed
  aperture, a trace cap of 40 per tile (the cap is active), small tiles;
* ``c2``: tabulated v(z), more output times than input samples, normalised
  by fold with min_fold 2;
* ``c3``: dt 3 ms (the index division is not a power of two), fractional
  t_min, 45 deg grid, a decreasing gradient V, an 85 deg angle limit, cap 60.

For each case it stores the inputs (the parameters as ``cases_json``), the
reference's V_rms at the input times, and the image and fold.  The reference
is imported through the namespace shim of ``make_golden.py``; nothing is
written into its tree.
"""
from __future__ import annotations

import importlib
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import import_reference  # noqa: E402

CASES = {
    "c0": dict(seed=11, n_tr=180, n_s=120, n_il=12, n_xl=10, il_spacing=25.0, xl_spacing=20.0,
               origin=(1000.0, 2000.0), azimuth_deg=0.0, dt_ms=4.0, t_min_ms=0.0, n_times=100,
               vel=("constant", 2000.0, 0.0), max_aperture_m=600.0, max_angle_deg=60.0,
               tile_size=100, max_traces_per_tile=5000, tda=True, normalize=False, min_fold=1),
    "c1": dict(seed=12, n_tr=220, n_s=100, n_il=9, n_xl=14, il_spacing=20.0, xl_spacing=25.0,
               origin=(500.0, -300.0), azimuth_deg=30.0, dt_ms=4.0, t_min_ms=40.0, n_times=90,
               vel=("gradient", 1800.0, 0.6), max_aperture_m=450.0, max_angle_deg=55.0,
               tile_size=16, max_traces_per_tile=40, tda=False, normalize=False, min_fold=1),
    "c2": dict(seed=13, n_tr=150, n_s=80, n_il=8, n_xl=8, il_spacing=30.0, xl_spacing=30.0,
               origin=(0.0, 0.0), azimuth_deg=0.0, dt_ms=2.0, t_min_ms=0.0, n_times=110,
               vel=("file", 1600.0, 0.0), max_aperture_m=500.0, max_angle_deg=65.0,
               tile_size=100, max_traces_per_tile=5000, tda=True, normalize=True, min_fold=2),
    "c3": dict(seed=14, n_tr=160, n_s=90, n_il=7, n_xl=11, il_spacing=22.5, xl_spacing=17.5,
               origin=(-340.25, 812.5), azimuth_deg=45.0, dt_ms=3.0, t_min_ms=6.5, n_times=95,
               vel=("gradient", 2100.0, -0.3), max_aperture_m=700.0, max_angle_deg=85.0,
               tile_size=30, max_traces_per_tile=60, tda=True, normalize=False, min_fold=1),
}

FILE_Z = np.array([0.0, 150.0, 400.0, 900.0, 2000.0], np.float32)
FILE_V = np.array([1600.0, 1750.0, 2100.0, 2600.0, 3300.0], np.float32)


def survey(c):
    """Seeded traces and geometry: midpoints over the grid and a margin."""
    rs = np.random.RandomState(c["seed"])
    n_tr = c["n_tr"]
    az = np.radians(c["azimuth_deg"])
    ext_il = c["n_il"] * c["il_spacing"]
    ext_xl = c["n_xl"] * c["xl_spacing"]
    u = rs.uniform(-0.15, 1.15, n_tr) * ext_il
    w = rs.uniform(-0.15, 1.15, n_tr) * ext_xl
    mx = c["origin"][0] + u * np.cos(az) - w * np.sin(az)
    my = c["origin"][1] + u * np.sin(az) + w * np.cos(az)
    off = rs.uniform(0.0, 500.0, n_tr)
    phi = rs.uniform(0.0, 2 * np.pi, n_tr)
    sx = (mx - 0.5 * off * np.cos(phi)).astype(np.float32)
    sy = (my - 0.5 * off * np.sin(phi)).astype(np.float32)
    rx = (mx + 0.5 * off * np.cos(phi)).astype(np.float32)
    ry = (my + 0.5 * off * np.sin(phi)).astype(np.float32)
    tr = rs.standard_normal((c["n_s"], n_tr)).astype(np.float32)
    return tr, sx, sy, rx, ry


def main(ref_root: str):
    eng, _, _, _, _, _ = import_reference(ref_root)
    evm = importlib.import_module("processors.migration.velocity_model")
    torch.manual_seed(0)
    out = {"file_z": FILE_Z, "file_v": FILE_V, "cases_json": np.array(json.dumps(CASES))}
    for name, c in CASES.items():
        tr, sx, sy, rx, ry = survey(c)
        kind, v0, k = c["vel"]
        if kind == "file":
            vm = evm.VelocityModel(velocity_type="file", v0=float(FILE_V[0]),
                                   velocity_array=FILE_V, z_axis=FILE_Z)
        else:
            vm = evm.VelocityModel(velocity_type=kind, v0=v0, gradient=k)
        t_in = torch.arange(c["n_s"], dtype=torch.float32) * c["dt_ms"]
        v_in = np.asarray(vm.rms_velocity_at_time(t_in), np.float32)
        e = eng.MigrationEngine(device=torch.device("cpu"))
        img, fold = e.migrate_bin_time_domain_rms(
            traces=tr, source_x=sx, source_y=sy, receiver_x=rx, receiver_y=ry,
            origin_x=c["origin"][0], origin_y=c["origin"][1], il_spacing=c["il_spacing"],
            xl_spacing=c["xl_spacing"], azimuth_deg=c["azimuth_deg"], n_il=c["n_il"],
            n_xl=c["n_xl"], dt_ms=c["dt_ms"], t_min_ms=c["t_min_ms"], n_times=c["n_times"],
            velocity_model=vm, max_aperture_m=c["max_aperture_m"],
            max_angle_deg=c["max_angle_deg"], tile_size=c["tile_size"],
            max_traces_per_tile=c["max_traces_per_tile"], normalize=c["normalize"],
            min_fold=c["min_fold"], use_time_dependent_aperture=c["tda"])
        out.update({f"{name}_traces": tr, f"{name}_sx": sx, f"{name}_sy": sy,
                    f"{name}_rx": rx, f"{name}_ry": ry, f"{name}_v_in": v_in,
                    f"{name}_image": np.asarray(img, np.float32),
                    f"{name}_fold": np.asarray(fold, np.float32)})
        print(name, "fold sum", float(np.sum(fold)), "image rms", float(np.sqrt(np.mean(img ** 2))))
    np.savez_compressed(os.path.join(HERE, "time_domain_rms.npz"), **out)
    print("wrote", os.path.join(HERE, "time_domain_rms.npz"))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SEISPROC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the SeisProc checkout> "
                 "(or set SEISPROC_REFERENCE)")
    main(ref)
