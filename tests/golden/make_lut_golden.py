"""Golden vectors for the KirchhoffMigrator's default traveltime lookup table,
made by running the reference itself (processors/migration/kirchhoff_migrator.py
with use_traveltime_lut=True, its default; traveltime_lut.py:77-308).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_lut_golden.py /path/to/reference

Writes ``migrator_lut.npz``: a mini gather migrated with a constant velocity and
with a linear-gradient v(z) (the table's curved-ray branch), plus a few table
lookups of the reference TraveltimeLUT.  The reference is imported through the
shim of ``make_golden.py``; nothing is written into its tree.
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from make_golden import import_reference  # noqa: E402
from seisproc_b200 import synthetic  # noqa: E402


def main(ref_root: str):
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    eng, kmig, cfg, vel, geo, sd = import_reference(ref_root)
    lutm = importlib.import_module("processors.migration.traveltime_lut")
    gs = synthetic.survey_3d(n_traces=300, seed=9, n_samples=100, extent=600.0, max_offset=400.0,
                             n_il=6, n_xl=5, spacing=30.0, n_diffractors=4, aperture=250.0,
                             lateral_velocity=False)
    grid = cfg.OutputGrid(n_time=90, n_inline=6, n_xline=5, dt=0.004, d_inline=30.0,
                          d_xline=30.0, t0=0.0, x_origin=gs.origin_x, y_origin=gs.origin_y)
    mcfg = cfg.MigrationConfig(output_grid=grid, max_aperture_m=250.0, max_angle_deg=55.0)
    gtr = gs.traces.cpu().numpy().astype(np.float32)
    gather = sd.SeismicData(traces=gtr, sample_rate=4.0)
    geom = geo.MigrationGeometry(source_x=gs.source_x, source_y=gs.source_y,
                                 receiver_x=gs.receiver_x, receiver_y=gs.receiver_y)
    out = dict(traces=gtr, source_x=geom.source_x, source_y=geom.source_y,
               receiver_x=geom.receiver_x, receiver_y=geom.receiver_y,
               grid=np.array([gs.origin_x, gs.origin_y, 30.0, 30.0, 6, 5, 4.0, 0.0, 1900.0,
                              250.0, 55.0, 90, 0.004], dtype=np.float64))
    models = {"constant": vel.create_constant_velocity(1900.0),
              "gradient": vel.create_linear_gradient_velocity(1800.0, 900.0, 2.0, 0.004)}
    for name, vm in models.items():
        mig = kmig.KirchhoffMigrator(vm, mcfg, device=torch.device("cpu"))
        assert mig.traveltime_lut is not None and mig.traveltime_lut._built
        img, fold = mig.migrate_gather(gather, geom)
        out[f"image_{name}"] = img.numpy()
        out[f"fold_{name}"] = fold.numpy()
        out[f"v0_{name}"] = np.float64(vm.v0)
        out[f"gradient_{name}"] = np.float64(getattr(vm, "gradient", 0.0) or 0.0)
        t = mig.traveltime_lut
        out[f"lut_{name}"] = np.array([t._max_offset, t._max_depth, t._n_offsets, t._n_depths],
                                      np.float64)
        rs = np.random.RandomState(4)
        h = rs.uniform(0, t._max_offset * 1.1, 200).astype(np.float32)
        z = rs.uniform(0, t._max_depth * 1.1, 200).astype(np.float32)
        out[f"probe_h_{name}"], out[f"probe_z_{name}"] = h, z
        out[f"probe_t_{name}"] = t.lookup_batch(torch.from_numpy(h), torch.from_numpy(z)).numpy()
    np.savez_compressed(os.path.join(HERE, "migrator_lut.npz"), **out)
    print("wrote", os.path.join(HERE, "migrator_lut.npz"), sorted(out))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SEISPROC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the SeisProc checkout> "
                 "(or set SEISPROC_REFERENCE)")
    main(ref)
