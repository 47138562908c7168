"""Device V_rms grids (pstm_velocity_grid) against the reference's scipy
interpolation (golden vectors) and the host float64 path, and a migration fed
a 3-D velocity model through the engine, on the GPU."""
import os

import numpy as np
import pytest
import torch

from conftest import ROOT

pytestmark = pytest.mark.gpu

G = np.load(os.path.join(ROOT, "tests", "golden", "velocity_io.npz"))


def _models():
    from seisproc_b200 import models as M
    return (M.create_2d_velocity(G["m_cube"][:, :, 1], G["m_z"], G["m_x"]),
            M.create_3d_velocity(G["m_cube"], G["m_z"], G["m_x"], G["m_y"]))


def _ulps(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64)).max()


def test_device_grid_matches_reference_points():
    """Output time i and output column i sit at golden point i: the grid's
    diagonal is the reference's scipy value at that point (extrapolated
    outside the axes)."""
    from seisproc_b200 import _lib
    from seisproc_b200.velocity_io import velocity_grid
    m2, m3 = _models()
    before = _lib.lib().pstm_launch_count()
    g3 = velocity_grid(m3, G["p_z"], G["p_x"], G["p_y"]).cpu().numpy()
    g2 = velocity_grid(m2, G["p_z"], G["p_x"]).cpu().numpy()
    assert _lib.lib().pstm_launch_count() - before == 2
    assert g3.shape == (G["p_z"].size, G["p_x"].size)
    assert _ulps(np.diag(g3), G["v3"]) <= 1
    assert _ulps(np.diag(g2), G["v2"]) <= 1


def test_device_grid_matches_host_path_on_a_survey_grid():
    from seisproc_b200.velocity_io import velocity_grid
    m2, m3 = _models()
    t = np.arange(1000) * 0.004
    il = np.arange(200)[:, None]
    xl = np.arange(200)[None, :]
    cx = (-150.0 + 9.0 * il + 0 * xl).ravel()
    cy = (-350.0 + 0 * il + 6.5 * xl).ravel()
    for m in (m2, m3):
        dev = velocity_grid(m, t, cx, cy)
        assert dev.is_cuda and dev.dtype == torch.float32 and dev.shape == (1000, 40000)
        host = m.rms_grid(t[::37], cx[::11], cy[::11])
        assert _ulps(dev.cpu().numpy()[::37, ::11], host) <= 1
    from seisproc_b200 import models as M
    v1 = velocity_grid(M.create_linear_gradient_velocity(1500.0, 500.0, 4.0), t, cx, cy)
    assert v1.shape == (1000,)


def test_engine_with_3d_velocity_model_equals_precomputed_grid():
    """migrate_bin_full(velocity_model=<3-D model>) resamples on the device;
    the image equals the one from the same V_rms grid passed as an array."""
    from seisproc_b200 import models as M
    from seisproc_b200 import synthetic
    from seisproc_b200.engine import MigrationEngine
    s = synthetic.survey_3d(n_traces=3000, seed=21, n_samples=200, extent=1000.0,
                            max_offset=800.0, n_il=9, n_xl=7, spacing=25.0, n_diffractors=6,
                            aperture=350.0)
    z = np.array([0.0, 0.3, 0.8], np.float32)
    x = np.array([s.origin_x - 100, s.origin_x + 400], np.float32)
    y = np.array([s.origin_y - 50, s.origin_y + 100, s.origin_y + 300], np.float32)
    cube = (1600 + 900 * z[:, None, None] + 0.1 * (x[None, :, None] - s.origin_x)
            + 0.2 * (y[None, None, :] - s.origin_y)).astype(np.float32)
    m3 = M.create_3d_velocity(cube, z, x, y)
    kw = dict(traces=s.traces.cpu().numpy(), source_x=s.source_x, source_y=s.source_y,
              receiver_x=s.receiver_x, receiver_y=s.receiver_y, origin_x=s.origin_x,
              origin_y=s.origin_y, il_spacing=s.il_spacing, xl_spacing=s.xl_spacing,
              azimuth_deg=0.0, n_il=s.n_il, n_xl=s.n_xl, dt_ms=s.dt_ms, t_min_ms=0.0,
              n_times=s.n_times, max_aperture_m=s.max_aperture_m,
              max_angle_deg=s.max_angle_deg, normalize=False)
    e = MigrationEngine()
    img_dev, fold_dev = e.migrate_bin_full(velocity_model=m3, **kw)
    il = np.arange(s.n_il)[:, None]
    xl = np.arange(s.n_xl)[None, :]
    cx = (s.origin_x + il * s.il_spacing + 0 * xl).ravel()
    cy = (s.origin_y + 0 * il + xl * s.xl_spacing).ravel()
    t_ms = np.arange(s.n_times, dtype=np.float32) * np.float32(s.dt_ms)
    grid = m3.rms_grid(np.asarray(t_ms, np.float64) / 1000.0, cx, cy)
    img_host, fold_host = e.migrate_bin_full(velocity_model=grid, **kw)
    assert np.array_equal(fold_dev, fold_host)
    err = np.linalg.norm(img_dev - img_host) / np.linalg.norm(img_host)
    assert err <= 1e-6, err
