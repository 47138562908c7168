"""Host-side logic that needs no GPU: backend selection, the config adapter's
contract with migrate_bin_full, models, grid/time inference, synthetic data."""
import inspect

import numpy as np
import pytest
import torch


def test_kernel_backend_selection():
    from seisproc_b200 import kernel_backend as kb
    assert kb.get_effective_backend() == kb.KernelBackend.CUDA_SM100
    assert kb.get_effective_backend("auto") == kb.KernelBackend.CUDA_SM100
    assert kb.get_effective_backend("cuda_sm100") == kb.KernelBackend.CUDA_SM100
    for bad in ("python", "metal_cpp", kb.KernelBackend.PYTHON):
        with pytest.raises(ValueError):
            kb.get_effective_backend(bad)
    with pytest.raises(ValueError):
        kb.get_effective_backend("opencl")
    kb.set_global_backend("python")
    try:
        with pytest.raises(ValueError):
            kb.get_effective_backend()
        assert kb.get_effective_backend("auto") == kb.KernelBackend.CUDA_SM100
    finally:
        kb.set_global_backend(kb.KernelBackend.AUTO)
    info = kb.get_backend_info()
    assert info["effective_backend"] == "cuda_sm100" and info["python_available"] is False


def test_no_cpu_fallback_without_cuda():
    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from seisproc_b200.engine import MigrationEngine
    with pytest.raises(RuntimeError, match="CUDA"):
        MigrationEngine()


def test_config_adapter_keys_match_engine_signature():
    """The reference asserts the adapter's keys are accepted by migrate_bin_full
    (tests/test_config_adapter.py:416-454)."""
    from seisproc_b200.config_adapter import ConfigAdapter
    from seisproc_b200.engine import MigrationEngine
    a = ConfigAdapter({"x_origin": 10.0, "y_origin": 20.0, "output_bin_il": 12.5,
                       "inline_min": 1, "inline_max": 40, "xline_min": 5, "xline_max": 24,
                       "dt_ms": 2.0, "time_min_ms": 0.0, "time_max_ms": 2000.0,
                       "velocity_v0": 2200.0, "max_aperture_m": 3000.0, "max_angle_deg": 50.0})
    z = np.zeros(3)
    p = a.get_engine_params(np.zeros((10, 3)), z, z, z, z)
    sig = inspect.signature(MigrationEngine.migrate_bin_full).parameters
    assert set(p) <= set(sig)
    assert p["n_il"] == 40 and p["n_xl"] == 20 and p["n_times"] == 1001
    assert p["il_spacing"] == 12.5 and p["xl_spacing"] == 25.0
    assert a.validate() == (True, "Configuration valid")
    bad = ConfigAdapter({"inline_min": 10, "inline_max": 1, "velocity_v0": -5})
    ok, msg = bad.validate()
    assert not ok and "inline range" in msg and "velocity" in msg


def test_migration_config_validation():
    from seisproc_b200 import models as M
    with pytest.raises(ValueError):
        M.MigrationConfig(max_angle_deg=95)
    with pytest.raises(ValueError):
        M.MigrationConfig(min_offset_m=10, max_offset_m=5)
    with pytest.raises(ValueError):
        M.OutputGrid(dt=0)
    c = M.MigrationConfig(weight_mode=M.WeightMode.FULL)
    c2 = M.MigrationConfig.from_dict(c.to_dict())
    assert c2.weight_mode == M.WeightMode.FULL and c2.output_grid == c.output_grid


def test_velocity_models():
    from seisproc_b200 import models as M
    from seisproc_b200 import velocity as V
    v = V.VelocityModel("constant", 2000.0)
    assert np.all(v.rms_velocity_at_time(np.array([0.0, 500.0])) == 2000.0)
    g = V.VelocityModel("gradient", 1500.0, gradient=0.5)
    r = g.rms_velocity_at_time(np.array([0.5, 1000.0]))
    assert r[0] == 1500.0 and r[1] > 1500.0
    t = np.linspace(0, 4, 41)
    cube = 1500.0 + 500.0 * t[:, None, None] + np.zeros((41, 3, 4))
    m = M.create_3d_velocity(cube, t, np.array([0.0, 100, 200]), np.array([0.0, 50, 100, 150]))
    assert m.velocity_type == M.VelocityType.V_OF_XYZ
    assert m.get_velocity_at(np.array([1.05]), np.array([37.0]), np.array([12.0]))[0] == \
        pytest.approx(1500 + 500 * 1.05, rel=1e-6)
    grid = m.rms_grid(np.array([0.0, 2.0]), np.array([0.0, 200.0]), np.array([0.0, 150.0]))
    assert grid.shape == (2, 2) and np.allclose(grid[1], 2500.0)
    tt, vi = M.rms_to_interval_velocity(t[1:], np.full(40, 2000.0))
    assert np.allclose(vi, 2000.0)
    _, vr = M.interval_to_rms_velocity(t[1:], np.full(40, 2000.0))
    assert np.allclose(vr, 2000.0)


def test_engine_velocity_at_outputs():
    from seisproc_b200.engine import velocity_at_outputs
    from seisproc_b200 import velocity as V
    t = np.arange(5, dtype=np.float32) * 4.0
    cx = np.zeros(6)
    assert velocity_at_outputs(2000.0, None, t, cx, cx).shape == (1,)
    assert velocity_at_outputs(0, V.VelocityModel("gradient", 1500, 0.5), t, cx, cx).shape == (5,)
    assert velocity_at_outputs(0, np.ones((5, 2, 3)), t, cx, cx).shape == (5, 6)


def test_regular_grid_inference():
    from seisproc_b200.kirchhoff import regular_grid_from_points, regular_times_from_depth
    il = np.arange(4)[:, None]
    xl = np.arange(3)[None, :]
    x = (100.0 + il * 12.5 + xl * 0.0).ravel()
    y = (50.0 + il * 0.0 + xl * 25.0).ravel()
    assert regular_grid_from_points(x, y, 4, 3) == (100.0, 50.0, 12.5, 0.0, 0.0, 25.0)
    with pytest.raises(ValueError):
        regular_grid_from_points(x + np.random.RandomState(0).rand(12) * 5, y, 4, 3)
    z = 2000.0 * (np.arange(10) * 4.0 / 1000.0) / 2.0
    assert regular_times_from_depth(z, 2000.0) == pytest.approx((0.0, 4.0))


def test_synthetic_noise_is_keyed_and_deterministic():
    from seisproc_b200 import synthetic
    ids = torch.arange(10, dtype=torch.int64)
    a = synthetic.hashed_gaussian(5, ids, 100)
    b = synthetic.hashed_gaussian(5, ids[3:], 100)
    assert torch.equal(a[:, 3:], b)
    assert abs(float(a.mean())) < 0.2 and 0.8 < float(a.std()) < 1.2
    s1 = synthetic.survey_2d(seed=1, n_offsets=2, n_cmp=16, n_samples=64, n_diffractors=3)
    s2 = synthetic.survey_2d(seed=1, n_offsets=2, n_cmp=16, n_samples=64, n_diffractors=3)
    assert torch.equal(s1.traces, s2.traces)
    c = synthetic.class_counts_loguniform()
    assert c.shape == (64,) and c.min() >= 2000 and c.max() <= 40000


def test_offset_taper_matches_reference_controller():
    """The migrator's per-trace offset taper against the reference's
    ApertureController._compute_offset_mask (golden vectors)."""
    import os
    from conftest import ROOT
    from seisproc_b200.migrator import offset_taper
    g = np.load(os.path.join(ROOT, "tests", "golden", "aperture_taper.npz"))
    off = np.hypot(g["rx"] - g["sx"], g["ry"] - g["sy"])
    for k in range(2):
        tw, _, _, omin, omax = g[f"params{k}"]
        assert np.allclose(offset_taper(off, omin, omax, tw), g[f"offset_mask{k}"], atol=2e-6)


def test_engine_trace_blocks():
    """A bin's blocks of traces tile it exactly; several blocks start with one
    an eighth of the bin (its upload is all the first launch waits for)."""
    from seisproc_b200.engine import MigrationEngine
    eng = MigrationEngine.__new__(MigrationEngine)  # no device needed for the split
    eng.block_traces, eng.max_blocks = 100_000, 4
    for n in (0, 5, 150_000, 200_000, 500_000, 1_000_003):
        blocks = eng._trace_blocks(n)
        assert blocks[0][0] == 0 and sum(c for _, c in blocks) == n
        assert all(a + c == b for (a, c), (b, _) in zip(blocks, blocks[1:]))
        assert len(blocks) == min(4, max(1, n // 100_000))
        if len(blocks) > 1:
            assert blocks[0][1] == n // (2 * len(blocks))
