"""Time-domain RMS operator, CPU side: the oracle against golden vectors from
the reference's migrate_bin_time_domain_rms, the host logic (midpoint columns,
tile trace lists, V_rms table) against the oracle, and the C entry point's
argument validation (no device work)."""
import ctypes as C
import json

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import time_domain as otd


def _cases():
    g = load_golden("time_domain_rms")
    return g, json.loads(str(g["cases_json"]))


def _velocity_model(g, c):
    from seisproc_b200.velocity import VelocityModel
    kind, v0, k = c["vel"]
    if kind == "file":
        return VelocityModel("file", float(g["file_v"][0]), velocity_array=g["file_v"],
                             z_axis=g["file_z"])
    return VelocityModel(kind, v0, gradient=k)


def _oracle(g, n, c, v_in=None):
    img, fold = otd.time_domain_rms_f32(
        g[n + "_traces"], g[n + "_sx"], g[n + "_sy"], g[n + "_rx"], g[n + "_ry"],
        g[n + "_v_in"] if v_in is None else v_in, c["origin"][0], c["origin"][1],
        c["il_spacing"], c["xl_spacing"], c["azimuth_deg"], c["n_il"], c["n_xl"], c["dt_ms"],
        c["t_min_ms"], c["n_times"], c["max_aperture_m"], c["max_angle_deg"], c["tile_size"],
        200, c["max_traces_per_tile"], c["tda"])
    if c["normalize"]:
        m = fold >= c["min_fold"]
        img = img.copy()
        img[m] = img[m] / fold[m]
    return img, fold


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "c3"])
def test_oracle_matches_reference_golden(name):
    g, cases = _cases()
    img, fold = _oracle(g, name, cases[name])
    np.testing.assert_array_equal(fold, g[name + "_fold"])
    assert rel_l2(img, g[name + "_image"]) < 1e-6
    assert g[name + "_fold"].sum() > 1000  # the case has contributions


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "c3"])
def test_velocity_table_matches_reference(name):
    """The engine VelocityModel's tensor branch gives the reference's float32
    V_rms at the input times, bit for bit."""
    g, cases = _cases()
    c = cases[name]
    t_in = 0.0 + torch.arange(c["n_s"], dtype=torch.float32) * c["dt_ms"]
    v = _velocity_model(g, c).rms_velocity_at_time(t_in)
    np.testing.assert_array_equal(v.numpy(), g[name + "_v_in"])
    if c["vel"][0] != "file":
        np.testing.assert_array_equal(
            otd.rms_velocity_torch_order_f32(c["vel"][0], c["vel"][1], c["vel"][2],
                                             t_in.numpy()), g[name + "_v_in"])


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "c3"])
def test_host_pairs_and_columns_match_oracle(name):
    from seisproc_b200 import time_domain as td
    g, cases = _cases()
    c = cases[name]
    t = {k: torch.from_numpy(g[f"{name}_{k}"]) for k in ("sx", "sy", "rx", "ry")}
    mid_x, mid_y, hoff, col = td.trace_geometry(t["sx"], t["sy"], t["rx"], t["ry"],
                                                c["origin"][0], c["origin"][1],
                                                c["il_spacing"], c["xl_spacing"],
                                                c["azimuth_deg"], c["n_il"], c["n_xl"])
    mx = (g[name + "_sx"] + g[name + "_rx"]) / np.float32(2)
    my = (g[name + "_sy"] + g[name + "_ry"]) / np.float32(2)
    np.testing.assert_array_equal(mid_x.numpy(), mx)
    il, xl = otd.trace_columns_f32(mx, my, c["origin"][0], c["origin"][1], c["il_spacing"],
                                   c["xl_spacing"], c["azimuth_deg"], c["n_il"], c["n_xl"])
    np.testing.assert_array_equal(col.numpy(), il * c["n_xl"] + xl)
    ox, oy = otd.output_grid_f32(c["origin"][0], c["origin"][1], c["il_spacing"],
                                 c["xl_spacing"], c["azimuth_deg"], c["n_il"], c["n_xl"])
    tile = td.effective_tile_size(c["tile_size"], c["max_traces_per_tile"], 200)
    assert tile == otd.effective_tile_size(c["tile_size"], c["max_traces_per_tile"], 200)
    p_tile, p_trace = td.tile_pairs(torch.from_numpy(ox), torch.from_numpy(oy), mid_x, mid_y,
                                    tile, c["max_aperture_m"], c["max_traces_per_tile"],
                                    elements=4096)
    want = {(i, int(j)) for i, (_, _, sel) in enumerate(
        otd.tile_trace_lists(ox, oy, mx, my, tile, c["max_aperture_m"],
                             c["max_traces_per_tile"])) for j in sel}
    got = set(zip(p_tile.tolist(), p_trace.tolist()))
    assert got == want
    if c["max_traces_per_tile"] < 1000:  # the cap bites in this case
        counts = np.bincount(p_tile.numpy())
        assert counts.max() == c["max_traces_per_tile"]


def test_effective_tile_size_follows_memory_bound():
    from seisproc_b200.time_domain import effective_tile_size
    assert effective_tile_size(100, 5000, 200) == 100
    assert effective_tile_size(1000, 5000, 200) == 322
    assert effective_tile_size(1000, 10 ** 6, 400) == 50


def test_entry_point_rejects_bad_arguments_without_device():
    from seisproc_b200 import _lib
    L = _lib.lib()
    fn = L.pstm_time_rms_migrate
    z = [None] * 9
    assert fn(None, *z[:9], 0, None, None, 0, None, None, None) == _lib.PSTM_EINVAL
    assert "params" in _lib.last_error()
    buf = (C.c_float * 4)()
    good = dict(n_samples=10, n_traces=1, n_points=1, n_times=2, tile=1, dt_ms=4.0,
                t_min_ms=0.0, max_aperture_m=100.0, max_angle_deg=60.0,
                time_dependent_aperture=1)
    for bad in (dict(n_samples=0), dict(n_times=0), dict(tile=0), dict(dt_ms=0.0),
                dict(n_points=0), dict(max_angle_deg=float("nan")), dict(n_times=30000)):
        p = _lib.TimeRmsParams(**{**good, **bad})
        st = fn(C.byref(p), *z[:9], 0, None, None, 0, C.cast(buf, C.c_void_p),
                C.cast(buf, C.c_void_p), None)
        assert st == _lib.PSTM_EINVAL, bad
    p = _lib.TimeRmsParams(**good)
    assert fn(C.byref(p), *z[:9], 0, None, None, 0, None, None, None) == _lib.PSTM_EINVAL
    # segments to process but NULL inputs
    assert fn(C.byref(p), *z[:9], 1, None, None, 1, C.cast(buf, C.c_void_p),
              C.cast(buf, C.c_void_p), None) == _lib.PSTM_EINVAL
    assert "NULL input" in _lib.last_error()


@pytest.mark.parametrize("name", ["c0", "c1", "c3"])
def test_column_pairs_sorted_by_midpoint_column(name):
    """The pair list the kernel takes: every selected (tile, trace) pair once,
    grouped by the trace's midpoint column, one segment per column."""
    from seisproc_b200 import time_domain as td
    g, cases = _cases()
    c = cases[name]
    t = {k: torch.from_numpy(g[f"{name}_{k}"]) for k in ("sx", "sy", "rx", "ry")}
    mid_x, mid_y, _, col = td.trace_geometry(t["sx"], t["sy"], t["rx"], t["ry"],
                                             c["origin"][0], c["origin"][1], c["il_spacing"],
                                             c["xl_spacing"], c["azimuth_deg"], c["n_il"],
                                             c["n_xl"])
    ox, oy = (torch.from_numpy(a) for a in otd.output_grid_f32(
        c["origin"][0], c["origin"][1], c["il_spacing"], c["xl_spacing"], c["azimuth_deg"],
        c["n_il"], c["n_xl"]))
    tile = td.effective_tile_size(c["tile_size"], c["max_traces_per_tile"], 200)
    args = (ox, oy, mid_x, mid_y)
    p_tile, p_trace = td.tile_pairs(*args, tile, c["max_aperture_m"], c["max_traces_per_tile"])
    pair_trace, pair_tile, seg_off, seg_col = td.column_pairs(
        *args, col, tile, c["max_aperture_m"], c["max_traces_per_tile"])
    assert pair_trace.dtype == torch.int32 and seg_off.dtype == torch.int64
    assert set(zip(pair_tile.tolist(), pair_trace.tolist())) == \
        set(zip(p_tile.tolist(), p_trace.tolist()))
    assert int(seg_off[0]) == 0 and int(seg_off[-1]) == pair_trace.numel()
    assert seg_off.numel() == seg_col.numel() + 1
    assert torch.all(seg_col[1:] > seg_col[:-1])  # one segment per column, ascending
    for g_ in range(seg_col.numel()):
        a, b = int(seg_off[g_]), int(seg_off[g_ + 1])
        assert b > a
        assert torch.all(col[pair_trace[a:b].long()] == seg_col[g_])


def test_config_adapter_time_domain_params():
    """ConfigAdapter.get_time_domain_params gives the reference's keys and
    values (its known answer, tests/test_time_domain_migration.py:362-402), and
    the batch worker's migrate_bin_time_domain_rms call built from them
    (views/migration_monitor_dialog.py:328-362) binds to the engine's signature."""
    import inspect
    from seisproc_b200.config_adapter import ConfigAdapter
    from seisproc_b200.engine import MigrationEngine
    from seisproc_b200.velocity import create_velocity_model
    a = ConfigAdapter({"x_origin": 100.0, "y_origin": 200.0, "output_bin_il": 25.0,
                       "output_bin_xl": 25.0, "inline_min": 1, "inline_max": 10,
                       "xline_min": 1, "xline_max": 10, "dt_ms": 4.0, "time_min_ms": 0.0,
                       "time_max_ms": 400.0, "velocity_v0": 2500.0, "max_aperture_m": 3000.0,
                       "max_angle_deg": 60.0, "tile_size": 100})
    z = np.zeros(50, np.float32)
    tr = np.zeros((101, 50), np.float32)
    params = a.get_time_domain_params(traces=tr, source_x=z, source_y=z, receiver_x=z,
                                      receiver_y=z)
    assert "n_times" in params and "tile_size" in params
    assert params["n_times"] == 101
    assert params["origin_x"] == 100.0 and params["origin_y"] == 200.0
    assert params["use_time_dependent_aperture"] is True
    p = a.params
    worker_kwargs = dict(
        traces=tr, source_x=z, source_y=z, receiver_x=z, receiver_y=z,
        **{k: params[k] for k in ("origin_x", "origin_y", "il_spacing", "xl_spacing",
                                  "azimuth_deg", "n_il", "n_xl", "dt_ms", "t_min_ms",
                                  "max_aperture_m", "max_angle_deg")},
        n_times=p.n_samples, velocity_model=create_velocity_model("gradient", 2500.0, 0.4),
        tile_size=p.tile_size, sample_batch_size=p.sample_batch_size,
        max_traces_per_tile=p.max_traces_per_tile, normalize=False,
        progress_callback=None, enable_profiling=True, use_time_dependent_aperture=True)
    inspect.signature(MigrationEngine.migrate_bin_time_domain_rms).bind(None, **worker_kwargs)


def test_config_adapter_advanced_fields_and_defaults():
    """The adapter's time-domain fields and their defaults, as the reference
    pins them (tests/test_time_domain_migration.py:331-430)."""
    from seisproc_b200.config_adapter import ConfigAdapter
    base = {"x_origin": 0.0, "y_origin": 0.0, "output_bin_il": 25.0, "output_bin_xl": 25.0,
            "inline_min": 1, "inline_max": 10, "xline_min": 1, "xline_max": 10, "dt_ms": 4.0,
            "time_min_ms": 0.0, "time_max_ms": 400.0, "velocity_v0": 2500.0,
            "max_aperture_m": 3000.0, "max_angle_deg": 60.0}
    p = ConfigAdapter({**base, "tile_size": 200, "use_time_domain": True, "use_kdtree": True,
                       "sample_batch_size": 150}).params
    assert p.tile_size == 200 and p.use_time_domain is True and p.use_kdtree is True
    assert p.sample_batch_size == 150
    p = ConfigAdapter(base).params
    assert p.tile_size == 100 and p.use_time_domain is False and p.use_kdtree is False
    assert p.sample_batch_size == 200 and p.max_traces_per_tile == 5000


def test_engine_velocity_model_known_answers():
    """V_rms(t) of the engine's velocity model on scalars, arrays and float32
    tensors, as the reference pins it (tests/test_velocity_model.py:95-150)."""
    from seisproc_b200.velocity import VelocityModel
    m = VelocityModel(velocity_type="gradient", v0=2000.0, gradient=0.5)
    v = [m.rms_velocity_at_time(t) for t in (500.0, 1000.0, 2000.0)]
    assert v[0] < v[1] < v[2]
    assert m.rms_velocity_at_time(0.0) == 2000.0
    t = torch.tensor([0.0, 500.0, 1000.0, 2000.0], dtype=torch.float32)
    vt = m.rms_velocity_at_time(t)
    assert isinstance(vt, torch.Tensor) and vt.shape == (4,) and vt.dtype == torch.float32
    assert torch.isclose(vt[0], torch.tensor(2000.0))
    assert (vt[1:] > vt[:-1]).all()
    # the float32 tensor branch and the float64 array branch agree to rounding
    np.testing.assert_allclose(vt.numpy(), m.rms_velocity_at_time(t.numpy()), rtol=1e-6)
    z = VelocityModel(velocity_type="gradient", v0=2500.0, gradient=0.0)
    assert np.allclose(z.rms_velocity_at_time(np.array([0, 500, 1000, 2000])), 2500.0)
    assert torch.all(z.rms_velocity_at_time(t) == 2500.0)
    s = VelocityModel(velocity_type="gradient", v0=1500.0, gradient=0.5)
    assert 1500.0 < s.rms_velocity_at_time(2000.0) < 2500.0


@pytest.mark.parametrize("name", ["c0", "c1", "c2", "c3"])
def test_torch_port_bit_identical_to_reference(name):
    """The oracle's torch port of the reference's loop reproduces the
    reference's image and fold bit for bit (same float32 operations, same
    cap selection, same scatter order)."""
    g, cases = _cases()
    c = cases[name]
    ox, oy = otd.output_grid_f32(c["origin"][0], c["origin"][1], c["il_spacing"],
                                 c["xl_spacing"], c["azimuth_deg"], c["n_il"], c["n_xl"])
    img, fold = otd.time_domain_rms_torch_port(
        g[name + "_traces"], g[name + "_sx"], g[name + "_sy"], g[name + "_rx"],
        g[name + "_ry"], ox, oy, c["n_times"], g[name + "_v_in"], c["dt_ms"], c["t_min_ms"],
        c["max_aperture_m"], c["max_angle_deg"], c["n_il"], c["n_xl"], c["origin"][0],
        c["origin"][1], c["il_spacing"], c["xl_spacing"], c["azimuth_deg"], c["tile_size"],
        200, c["max_traces_per_tile"], c["tda"])
    img, fold = img.numpy(), fold.numpy()
    if c["normalize"]:
        m = fold >= c["min_fold"]
        img = img.copy()
        img[m] = img[m] / fold[m]
    np.testing.assert_array_equal(fold, g[name + "_fold"])
    np.testing.assert_array_equal(img, g[name + "_image"])


def test_oracles_agree_up_to_torch_sqrt_rounding():
    """The numpy float32 restatement (IEEE square roots) and the torch port of
    the reference (torch's CPU float32 sqrt, an ulp off on ~0.7 % of inputs)
    agree on a 3000-trace case with the cap active except where that ulp in
    t_out straddles an integer output index: a few dozen of 4e7 fold counts."""
    rs = np.random.RandomState(5)
    n_tr, n_s, n_il, n_xl, sp, az = 3000, 300, 24, 20, 25.0, 20.0
    u = rs.uniform(-0.1, 1.1, n_tr) * n_il * sp
    w = rs.uniform(-0.1, 1.1, n_tr) * n_xl * sp
    a = np.radians(az)
    mx, my = u * np.cos(a) - w * np.sin(a), u * np.sin(a) + w * np.cos(a)
    off, phi = rs.uniform(0, 500, n_tr), rs.uniform(0, 2 * np.pi, n_tr)
    sx, sy = (mx - 0.5 * off * np.cos(phi)).astype(np.float32), (my - 0.5 * off * np.sin(phi)).astype(np.float32)
    rx, ry = (mx + 0.5 * off * np.cos(phi)).astype(np.float32), (my + 0.5 * off * np.sin(phi)).astype(np.float32)
    tr = rs.standard_normal((n_s, n_tr)).astype(np.float32)
    v = otd.rms_velocity_torch_order_f32("gradient", 1700.0, 0.5,
                                         np.arange(n_s, dtype=np.float32) * np.float32(4.0))
    ox, oy = otd.output_grid_f32(0, 0, sp, sp, az, n_il, n_xl)
    i1, f1 = otd.time_domain_rms_f32(tr, sx, sy, rx, ry, v, 0, 0, sp, sp, az, n_il, n_xl, 4.0,
                                     8.0, 280, 400.0, 50.0, tile_size=40, max_traces_per_tile=300)
    i2, f2 = otd.time_domain_rms_torch_port(tr, sx, sy, rx, ry, ox, oy, 280, v, 4.0, 8.0, 400.0,
                                            50.0, n_il, n_xl, 0, 0, sp, sp, az, tile_size=40,
                                            max_traces_per_tile=300)
    f2, i2 = f2.numpy(), i2.numpy()
    assert f1.sum() > 3e7
    assert (f1 != f2).sum() <= 60 and np.abs(f1 - f2).max() <= 2
    assert rel_l2(i2, i1) < 3e-4
