"""Time-domain RMS operator on the GPU (pstm_time_rms_migrate) against the
reference's own results (golden vectors) and the float32 oracle.

The output index of every contribution is the reference's float32 expression
with IEEE rounding, so folds agree except where a rounding the reference takes
differently moves one count: torch's CPU float32 sqrt (not correctly rounded
on every input) across an integer index, or an arctangent an ulp apart at the
angle limit -- at most a few entries per case.  The
image is compared where the folds agree, with a float32 summation-order
tolerance of 1e-5 relative L2."""
import ctypes as C
import json

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import time_domain as otd

pytestmark = pytest.mark.gpu


def _vm(g, c):
    from seisproc_b200.velocity import VelocityModel
    kind, v0, k = c["vel"]
    if kind == "file":
        return VelocityModel("file", float(g["file_v"][0]), velocity_array=g["file_v"],
                             z_axis=g["file_z"])
    return VelocityModel(kind, v0, gradient=k)


def _compare(img, fold, want_img, want_fold, max_flips=2, tol=1e-5):
    diff = fold != want_fold
    assert diff.sum() <= max_flips, int(diff.sum())
    assert np.abs(fold - want_fold).max() <= 1
    keep = ~diff
    assert rel_l2(img[keep], want_img[keep]) < tol


def _engine_run(g, name, c, **over):
    from seisproc_b200.engine import MigrationEngine
    kw = dict(traces=g[name + "_traces"], source_x=g[name + "_sx"], source_y=g[name + "_sy"],
              receiver_x=g[name + "_rx"], receiver_y=g[name + "_ry"], origin_x=c["origin"][0],
              origin_y=c["origin"][1], il_spacing=c["il_spacing"], xl_spacing=c["xl_spacing"],
              azimuth_deg=c["azimuth_deg"], n_il=c["n_il"], n_xl=c["n_xl"], dt_ms=c["dt_ms"],
              t_min_ms=c["t_min_ms"], n_times=c["n_times"], velocity_model=_vm(g, c),
              max_aperture_m=c["max_aperture_m"], max_angle_deg=c["max_angle_deg"],
              tile_size=c["tile_size"], max_traces_per_tile=c["max_traces_per_tile"],
              normalize=c["normalize"], min_fold=c["min_fold"],
              use_time_dependent_aperture=c["tda"])
    kw.update(over)
    return MigrationEngine().migrate_bin_time_domain_rms(**kw)


@pytest.mark.parametrize("name", ["c0", "c1", "c2"])
def test_engine_matches_reference_golden(name):
    g = load_golden("time_domain_rms")
    c = json.loads(str(g["cases_json"]))[name]
    calls = []
    img, fold = _engine_run(g, name, c, progress_callback=lambda f, m: calls.append(f))
    assert img.shape == (c["n_times"], c["n_il"], c["n_xl"]) and img.dtype == np.float32
    _compare(img, fold, g[name + "_image"], g[name + "_fold"])
    assert calls[0] == 0.0 and calls[-1] == 1.0


def _survey(seed, n_tr, n_s, n_il, n_xl, spacing, az_deg=0.0, spread=500.0):
    rs = np.random.RandomState(seed)
    az = np.radians(az_deg)
    u = rs.uniform(-0.1, 1.1, n_tr) * n_il * spacing
    w = rs.uniform(-0.1, 1.1, n_tr) * n_xl * spacing
    mx, my = u * np.cos(az) - w * np.sin(az), u * np.sin(az) + w * np.cos(az)
    off, phi = rs.uniform(0, spread, n_tr), rs.uniform(0, 2 * np.pi, n_tr)
    geo = [(mx - 0.5 * off * np.cos(phi)), (my - 0.5 * off * np.sin(phi)),
           (mx + 0.5 * off * np.cos(phi)), (my + 0.5 * off * np.sin(phi))]
    tr = rs.standard_normal((n_s, n_tr)).astype(np.float32)
    return tr, [a.astype(np.float32) for a in geo]


def test_kernel_matches_oracle_with_trace_cap_and_gradient():
    """A larger case than the golden ones: 3000 traces, 40-point tiles, the
    300-trace cap active in most tiles, gradient V, rotated grid."""
    from seisproc_b200.engine import MigrationEngine
    from seisproc_b200.velocity import VelocityModel
    n_s, n_times, n_il, n_xl, sp, dt = 300, 280, 24, 20, 25.0, 4.0
    tr, (sx, sy, rx, ry) = _survey(5, 3000, n_s, n_il, n_xl, sp, az_deg=20.0)
    vm = VelocityModel("gradient", 1700.0, gradient=0.5)
    args = dict(origin_x=0.0, origin_y=0.0, il_spacing=sp, xl_spacing=sp, azimuth_deg=20.0,
                n_il=n_il, n_xl=n_xl, dt_ms=dt, t_min_ms=8.0, n_times=n_times,
                max_aperture_m=400.0, max_angle_deg=50.0)
    img, fold = MigrationEngine().migrate_bin_time_domain_rms(
        tr, sx, sy, rx, ry, velocity_model=vm, tile_size=40, max_traces_per_tile=300,
        normalize=False, use_time_dependent_aperture=True, **args)
    v_in = vm.rms_velocity_at_time(torch.arange(n_s, dtype=torch.float32) * dt).numpy()
    want_img, want_fold = otd.time_domain_rms_f32(
        tr, sx, sy, rx, ry, v_in, args["origin_x"], args["origin_y"], sp, sp, 20.0, n_il, n_xl,
        dt, 8.0, n_times, 400.0, 50.0, tile_size=40, max_traces_per_tile=300,
        use_time_dependent_aperture=True)
    assert want_fold.sum() > 1e5
    _compare(img, fold, want_img, want_fold, max_flips=4)


def test_linearity_in_the_traces():
    """migrate(a d1 + d2) = a migrate(d1) + migrate(d2), same fold."""
    from seisproc_b200.engine import MigrationEngine
    from seisproc_b200.velocity import VelocityModel
    tr1, geo = _survey(8, 4000, 400, 30, 30, 20.0)
    tr2 = np.random.RandomState(9).standard_normal(tr1.shape).astype(np.float32)
    e = MigrationEngine()
    kw = dict(origin_x=0.0, origin_y=0.0, il_spacing=20.0, xl_spacing=20.0, azimuth_deg=0.0,
              n_il=30, n_xl=30, dt_ms=4.0, t_min_ms=0.0, n_times=400,
              velocity_model=VelocityModel("constant", 2200.0), max_aperture_m=500.0,
              max_angle_deg=60.0, normalize=False)
    i1, f1 = e.migrate_bin_time_domain_rms(tr1, *geo, **kw)
    i2, f2 = e.migrate_bin_time_domain_rms(tr2, *geo, **kw)
    i3, f3 = e.migrate_bin_time_domain_rms((2.5 * tr1 + tr2).astype(np.float32), *geo, **kw)
    np.testing.assert_array_equal(f1, f2)
    np.testing.assert_array_equal(f1, f3)
    assert f1.sum() > 1e6
    assert rel_l2(i3, 2.5 * i1.astype(np.float64) + i2) < 1e-5


def test_no_contributions_gives_zeros():
    """Traces far outside the grid's aperture, and an empty survey."""
    from seisproc_b200.engine import MigrationEngine
    from seisproc_b200.velocity import VelocityModel
    tr, (sx, sy, rx, ry) = _survey(3, 50, 64, 5, 5, 25.0)
    kw = dict(origin_x=0.0, origin_y=0.0, il_spacing=25.0, xl_spacing=25.0, azimuth_deg=0.0,
              n_il=5, n_xl=5, dt_ms=4.0, t_min_ms=0.0, n_times=64,
              velocity_model=VelocityModel("constant", 2000.0), max_aperture_m=300.0,
              max_angle_deg=60.0, normalize=True)
    far = [a + np.float32(1e5) for a in (sx, sy, rx, ry)]
    img, fold = MigrationEngine().migrate_bin_time_domain_rms(tr, *far, **kw)
    assert not img.any() and not fold.any()
    e = np.zeros(0, np.float32)
    img, fold = MigrationEngine().migrate_bin_time_domain_rms(np.zeros((64, 0), np.float32),
                                                              e, e, e, e, **kw)
    assert img.shape == (64, 5, 5) and not img.any() and not fold.any()


def test_entry_point_overwrites_outputs_when_there_are_no_pairs():
    from seisproc_b200 import _lib
    image = torch.full((7, 12), 3.0, device="cuda")
    fold = torch.full((7, 12), 3.0, device="cuda")
    p = _lib.TimeRmsParams(n_samples=16, n_traces=0, n_points=12, n_times=7, tile=4, dt_ms=4.0,
                           t_min_ms=0.0, max_aperture_m=100.0, max_angle_deg=60.0,
                           time_dependent_aperture=1)
    st = _lib.lib().pstm_time_rms_migrate(
        C.byref(p), *([None] * 9), 0, None, None, 0, image.data_ptr(), fold.data_ptr(),
        torch.cuda.current_stream().cuda_stream)
    assert st == _lib.PSTM_OK
    assert not image.any().item() and not fold.any().item()
