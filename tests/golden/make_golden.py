"""Generate the golden fixtures by running the reference PSTM itself.

Run in a container where the reference source tree is available:

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /path/to/reference

The reference's ``processors``/``models`` package ``__init__`` files pull in GUI
and storage dependencies (PyQt6, zarr) that the migration code does not use,
so the script registers those directories as bare namespace packages and stubs
the storage modules before importing
``processors.migration.migration_engine`` and
``processors.migration.kirchhoff_migrator``.  Nothing is written into the
reference tree.

Each fixture stores the exact float32 inputs the reference saw and its outputs.
The full-size 2D workload (2880 traces x 501 samples) stores only its outputs
plus a SHA-256 of the regenerated float32 input, to keep the repository small.
"""
from __future__ import annotations

import hashlib
import importlib
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from seisproc_b200 import synthetic  # noqa: E402


def import_reference(ref_root: str):
    sys.dont_write_bytecode = True
    for pkg in ("processors", "models", "utils", "seisio"):
        m = types.ModuleType(pkg)
        m.__path__ = [os.path.join(ref_root, pkg)]
        sys.modules[pkg] = m
    m = types.ModuleType("processors.migration")
    m.__path__ = [os.path.join(ref_root, "processors", "migration")]
    sys.modules["processors.migration"] = m
    for stub in ("zarr", "segyio", "pywt", "numcodecs"):
        sys.modules.setdefault(stub, types.ModuleType(stub))
    eng = importlib.import_module("processors.migration.migration_engine")
    kmig = importlib.import_module("processors.migration.kirchhoff_migrator")
    cfg = importlib.import_module("models.migration_config")
    vel = importlib.import_module("models.velocity_model")
    geo = importlib.import_module("models.migration_geometry")
    sd = importlib.import_module("models.seismic_data")
    return eng, kmig, cfg, vel, geo, sd


def sha_f32(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def run_engine(eng, s: synthetic.Survey, tda=False, n_times=None, t_min_ms=None):
    e = eng.MigrationEngine(device=torch.device("cpu"))
    tr = s.traces.cpu().numpy()
    img, fold = e.migrate_bin_full(
        traces=tr, source_x=s.source_x, source_y=s.source_y, receiver_x=s.receiver_x,
        receiver_y=s.receiver_y, origin_x=s.origin_x, origin_y=s.origin_y,
        il_spacing=s.il_spacing, xl_spacing=s.xl_spacing, azimuth_deg=0.0, n_il=s.n_il,
        n_xl=s.n_xl, dt_ms=s.dt_ms, t_min_ms=s.t_min_ms if t_min_ms is None else t_min_ms,
        n_times=n_times if n_times is not None else s.n_times, velocity_mps=s.velocity_mps,
        max_aperture_m=s.max_aperture_m, max_angle_deg=s.max_angle_deg, normalize=False,
        use_time_dependent_aperture=tda)
    return tr, img, fold


def survey_inputs(s: synthetic.Survey, tr):
    return dict(traces=tr.astype(np.float32),
                source_x=s.source_x.astype(np.float32), source_y=s.source_y.astype(np.float32),
                receiver_x=s.receiver_x.astype(np.float32),
                receiver_y=s.receiver_y.astype(np.float32),
                grid=np.array([s.origin_x, s.origin_y, s.il_spacing, s.xl_spacing, s.n_il, s.n_xl,
                               s.dt_ms, s.t_min_ms, s.velocity_mps, s.max_aperture_m,
                               s.max_angle_deg], dtype=np.float64))


def main(ref_root: str, only=()):
    """Regenerates every fixture, or those named in ``only``."""
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    eng, kmig, cfg, vel, geo, sd = import_reference(ref_root)
    out = {}

    def want(name):
        return not only or name in only

    # 1. small 2D common-offset case (3 offsets x 48 CMPs x 251 samples)
    s = synthetic.survey_2d(seed=11, n_offsets=3, n_cmp=48, n_samples=251, n_diffractors=8)
    s.max_aperture_m = 400.0
    if want("full_2d_small"):
        tr, img, fold = run_engine(eng, s)
        np.savez_compressed(os.path.join(HERE, "full_2d_small.npz"), image=img, fold=fold,
                            **survey_inputs(s, tr), n_times=np.int64(s.n_times), tda=np.int64(0))
        out["full_2d_small"] = float(np.abs(img).max())

    # 2. same data, time-dependent aperture, shifted time origin, fewer output samples
    if want("full_2d_tda_tmin"):
        tr, img, fold = run_engine(eng, s, tda=True, n_times=200, t_min_ms=40.0)
        inp = survey_inputs(s, tr)
        inp["grid"][7] = 40.0
        np.savez_compressed(os.path.join(HERE, "full_2d_tda_tmin.npz"), image=img, fold=fold,
                            **inp, n_times=np.int64(200), tda=np.int64(1))
        out["full_2d_tda_tmin"] = float(np.abs(img).max())

    # 3. mini 3D survey, constant velocity (the reference takes a constant V only)
    if want("full_3d_mini"):
        s3 = synthetic.survey_3d(n_traces=800, seed=5, n_samples=128, extent=800.0,
                                 max_offset=500.0, n_il=8, n_xl=8, spacing=25.0, n_diffractors=6,
                                 aperture=300.0, lateral_velocity=False)
        s3.velocity_mps = 1800.0
        tr, img, fold = run_engine(eng, s3)
        np.savez_compressed(os.path.join(HERE, "full_3d_mini.npz"), image=img, fold=fold,
                            **survey_inputs(s3, tr), n_times=np.int64(s3.n_times),
                            tda=np.int64(0))
        out["full_3d_mini"] = float(np.abs(img).max())

    # 4. KirchhoffMigrator (direct DSR, no LUT) on a mini gather
    if want("migrator_mini"):
        gs = synthetic.survey_3d(n_traces=300, seed=9, n_samples=100, extent=600.0,
                                 max_offset=400.0, n_il=6, n_xl=5, spacing=30.0, n_diffractors=4,
                                 aperture=250.0, lateral_velocity=False)
        grid = cfg.OutputGrid(n_time=90, n_inline=6, n_xline=5, dt=0.004, d_inline=30.0,
                              d_xline=30.0, t0=0.0, x_origin=gs.origin_x, y_origin=gs.origin_y)
        mcfg = cfg.MigrationConfig(output_grid=grid, max_aperture_m=250.0, max_angle_deg=55.0)
        vm = vel.create_constant_velocity(1900.0)
        mig = kmig.KirchhoffMigrator(vm, mcfg, device=torch.device("cpu"),
                                     use_traveltime_lut=False)
        gtr = gs.traces.cpu().numpy().astype(np.float32)
        gather = sd.SeismicData(traces=gtr, sample_rate=4.0)
        geom = geo.MigrationGeometry(source_x=gs.source_x, source_y=gs.source_y,
                                     receiver_x=gs.receiver_x, receiver_y=gs.receiver_y)
        mimg, mfold = mig.migrate_gather(gather, geom)
        np.savez_compressed(os.path.join(HERE, "migrator_mini.npz"), image=mimg.numpy(),
                            fold=mfold.numpy(), traces=gtr,
                            source_x=geom.source_x, source_y=geom.source_y,
                            receiver_x=geom.receiver_x, receiver_y=geom.receiver_y,
                            grid=np.array([gs.origin_x, gs.origin_y, 30.0, 30.0, 6, 5, 4.0, 0.0,
                                           1900.0, 250.0, 55.0, 90, 0.004], dtype=np.float64))
        out["migrator_mini"] = float(mimg.abs().max())

    # 5. the full-size 2D workload: outputs + SHA-256 of the regenerated input
    if want("full_2d_config"):
        s2 = synthetic.survey_2d(seed=1234)
        tr, img, fold = run_engine(eng, s2)
        np.savez_compressed(os.path.join(HERE, "full_2d_config.npz"), image=img, fold=fold,
                            input_sha256=np.array(sha_f32(tr)),
                            geom_sha256=np.array(sha_f32(np.stack([s2.source_x, s2.source_y,
                                                                   s2.receiver_x,
                                                                   s2.receiver_y]))))
        out["full_2d_config"] = float(np.abs(img).max())

    # 6. a larger 3D survey at full trace density around the grid: 20k traces x
    # 500 samples -> 16 x 16 x 500 at 25 m, 800 m aperture, constant V (the
    # reference takes a constant V only); outputs + SHA-256 of the regenerated
    # input (generated on the CPU, as the test regenerates it)
    if want("full_3d_20k"):
        s6 = survey_3d_20k()
        tr, img, fold = run_engine(eng, s6)
        np.savez_compressed(os.path.join(HERE, "full_3d_20k.npz"), image=img, fold=fold,
                            input_sha256=np.array(sha_f32(tr)),
                            geom_sha256=np.array(sha_f32(np.stack([s6.source_x, s6.source_y,
                                                                   s6.receiver_x,
                                                                   s6.receiver_y]))),
                            velocity_mps=np.float64(s6.velocity_mps))
        out["full_3d_20k"] = float(np.abs(img).max())
    print(out)


def survey_3d_20k() -> synthetic.Survey:
    """The full_3d_20k fixture's input (CPU generator, seed 31)."""
    s = synthetic.survey_3d(n_traces=20000, seed=31, n_samples=500, extent=2400.0,
                            max_offset=1500.0, n_il=16, n_xl=16, spacing=25.0, n_diffractors=24,
                            aperture=800.0, lateral_velocity=False)
    s.velocity_mps = 2200.0
    return s


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SEISPROC_REFERENCE")
    if not ref:
        sys.exit(f"usage: python {os.path.basename(__file__)} <path to the SeisProc checkout> "
                 "[fixture ...] (or set SEISPROC_REFERENCE)")
    main(ref, tuple(sys.argv[2:]))
