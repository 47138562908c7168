"""Velocity ingestion on the host: the readers against golden vectors from the
reference's utils/velocity_io.py, the 2-D / 3-D interpolation against the
reference VelocityModel (scipy, linear extrapolation), SEG-Y decoding against
known IBM words and round trips, and the host half (per-axis tables) of the
device resampler."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from seisproc_b200 import models as M
from seisproc_b200 import velocity_io as V

G = np.load(os.path.join(ROOT, "tests", "golden", "velocity_io.npz"))


@pytest.fixture(scope="module")
def files(tmp_path_factory):
    d = tmp_path_factory.mktemp("vel")
    out = {}
    for k in ("tv", "cdptv", "ilxltv", "mixed"):
        p = d / f"{k}.txt"
        p.write_text(str(G[f"text_{k}"]) + "\n")
        out[k] = str(p)
    return out


def test_format_detection_matches_reference(files):
    for k, p in files.items():
        assert V.detect_velocity_format(p).value == str(G[f"format_{k}"]), k


def test_text_readers_match_reference(files):
    m = V.read_velocity_text(files["tv"])
    assert np.array_equal(m.z_axis, G["tv_t"]) and np.array_equal(m.data, G["tv_v"])
    m = V.read_velocity_text(files["mixed"], delimiter=",", skip_header=1, time_unit="ms",
                             velocity_unit="km/s")
    assert np.array_equal(m.z_axis, G["mixed_t"]) and np.array_equal(m.data, G["mixed_v"])


def test_cdptv_reader_matches_reference(files):
    m = V.read_velocity_cdptv(files["cdptv"])
    assert m.velocity_type == M.VelocityType.V_OF_XZ
    assert np.array_equal(m.z_axis, G["cdptv_t"])
    assert np.array_equal(m.x_axis, G["cdptv_x"])
    assert np.array_equal(m.data, G["cdptv_v"])
    info = V.preview_velocity_file(files["cdptv"])
    assert [info.n_locations, info.n_time_samples, *info.cdp_range] == G["cdptv_preview"].tolist()
    _, v = V.get_velocity_at_cdp(m, 1175, np.array([0.0, 0.3, 1.234, 2.0, 3.9], np.float32))
    assert np.allclose(v, G["cdp1175_v"], rtol=1e-6, atol=0)
    with pytest.raises(ValueError):
        V.read_velocity_cdptv(files["tv"])


def test_ilxltv_paths(files):
    info = V.preview_velocity_file(files["ilxltv"])
    assert [info.n_locations, info.n_time_samples, *info.inline_range, *info.xline_range] == \
        G["ilxl_preview"].tolist()
    m = V.velocity_info_to_model(info)  # the reference keeps the inline axis only
    assert np.array_equal(m.z_axis, G["ilxl_t"]) and np.array_equal(m.x_axis, G["ilxl_x"])
    assert np.array_equal(m.data, G["ilxl_v"])
    m3 = V.read_velocity_ilxltv_3d(files["ilxltv"])  # the full cube
    assert m3.velocity_type == M.VelocityType.V_OF_XYZ
    t, il, xl = m3.z_axis, m3.x_axis, m3.y_axis
    assert il.tolist() == [100, 102, 104] and xl.tolist() == [10, 20, 30, 40]
    want = 1500 + 0.7 * 1000 * t[:, None, None] + 3 * (il[None, :, None] - 100) + \
        0.5 * xl[None, None, :]
    assert np.allclose(m3.data, want, rtol=0, atol=0.006)


def test_ilxltv_3d_needs_every_location(tmp_path):
    p = tmp_path / "holes.txt"
    p.write_text("1 1 0 1500\n1 1 1000 2000\n1 2 0 1500\n1 2 1000 2000\n2 1 0 1500\n"
                 "2 1 1000 2000\n")
    with pytest.raises(ValueError, match="locations"):
        V.read_velocity_ilxltv_3d(p)


def _ref_models():
    m3 = M.create_3d_velocity(G["m_cube"], G["m_z"], G["m_x"], G["m_y"])
    m2 = M.create_2d_velocity(G["m_cube"][:, :, 1], G["m_z"], G["m_x"])
    return m2, m3


def test_interpolation_matches_reference_scipy():
    m2, m3 = _ref_models()
    v3 = m3.get_velocity_at(G["p_z"], G["p_x"], G["p_y"])
    v2 = m2.get_velocity_at(G["p_z"], G["p_x"])
    # float64 blends in both; results rounded to float32 agree to 1 ulp
    assert np.allclose(v3, G["v3"], rtol=2.5e-7, atol=0)
    assert np.allclose(v2, G["v2"], rtol=2.5e-7, atol=0)


def _blend(model, tabs):
    """The device kernel's blend restated in numpy: the lateral (x, y) blend
    at both ends of the model's time interval, then the lerp in time."""
    iz, wz, ix, wx, iy, wy = tabs
    d = model.data.astype(np.float64)
    if d.ndim == 2:
        d = d[:, :, None]
        iy = np.zeros_like(ix)
        wy = np.zeros_like(wx)
    nz, nx, ny = d.shape
    dz1, dx1, dy1 = int(nz > 1), int(nx > 1), int(ny > 1)

    def lateral(rows):
        r = rows[:, None]
        return ((1 - wx) * (1 - wy) * d[r, ix, iy] + (1 - wx) * wy * d[r, ix, iy + dy1]
                + wx * (1 - wy) * d[r, ix + dx1, iy] + wx * wy * d[r, ix + dx1, iy + dy1])

    v0, v1 = lateral(iz), lateral(iz + dz1)
    return ((1 - wz)[:, None] * v0 + wz[:, None] * v1).astype(np.float32)


def test_axis_tables_reproduce_rms_grid():
    m2, m3 = _ref_models()
    t = np.linspace(-0.2, 4.0, 57)
    cx = np.linspace(-300.0, 2000.0, 23)
    cy = np.linspace(-400.0, 1000.0, 23)
    for m in (m2, m3):
        tabs = V.axis_tables(m, t, cx, cy)
        assert tabs[0].dtype == np.int32 and tabs[1].dtype == np.float64
        assert tabs[0].min() >= 0 and tabs[0].max() <= m.data.shape[0] - 2
        got = _blend(m, tabs)
        ref = m.rms_grid(t, cx, cy)
        assert np.allclose(got, ref, rtol=2.5e-7, atol=0)
    with pytest.raises(ValueError):
        V.axis_tables(M.create_constant_velocity(2000.0), t, cx, cy)


def test_ibm_float_known_words():
    # IBM single precision: 1.0 = 0x41100000, -118.625 = 0xC276A000, 0.15625 = 0x40280000
    w = np.array([0x41100000, 0xC276A000, 0x40280000, 0], np.uint32)
    x = np.array([1.0, -118.625, 0.15625, 0.0], np.float32)
    assert np.array_equal(V.ibm_to_ieee(w), x)
    assert np.array_equal(V.ieee_to_ibm(x), w)
    r = np.random.RandomState(3).uniform(-1e5, 1e5, 1000).astype(np.float32)
    back = V.ibm_to_ieee(V.ieee_to_ibm(r))
    assert np.all(np.abs(back - r) <= 2.0 ** -20 * np.abs(r))


def test_segy_round_trip_and_velocity_reader(tmp_path):
    rs = np.random.RandomState(8)
    tr = rs.uniform(1400, 4500, (5, 120)).astype(np.float32)
    for fmt in (1, 5):
        p = tmp_path / f"v{fmt}.sgy"
        V.write_segy_traces(p, tr, 4000, cdp=[500, 501, 502, 503, 504], inline=[7] * 5,
                            xline=[1, 2, 3, 4, 5], fmt=fmt, delay_ms=8)
        s = V.read_segy_traces(p)
        assert s["format"] == fmt and s["interval_us"] == 4000
        assert np.allclose(s["samples_ms"], 8 + 4.0 * np.arange(120))
        assert s["cdp"].tolist() == [500, 501, 502, 503, 504]
        assert s["xline"].tolist() == [1, 2, 3, 4, 5] and set(s["inline"]) == {7}
        tol = 0 if fmt == 5 else 2.0 ** -20
        assert np.all(np.abs(s["traces"] - tr) <= tol * np.abs(tr))
        m = V.read_velocity_segy(p)
        assert m.velocity_type == M.VelocityType.V_OF_XZ
        assert m.x_axis.tolist() == [500, 501, 502, 503, 504]
        assert np.allclose(m.z_axis, (8 + 4.0 * np.arange(120)) / 1000.0)
        info = V.preview_velocity_file(p)
        assert info.is_valid and info.cdp_range == (500, 504) and info.n_locations == 5
        assert V.velocity_info_to_model(info).data.shape == (120, 5)
    p = tmp_path / "one.segy"
    V.write_segy_traces(p, tr[:1], 2000)
    m = V.read_velocity_segy(p)
    assert m.velocity_type == M.VelocityType.V_OF_Z and m.z_axis.size == 120
    p = tmp_path / "nocdp.sgy"
    V.write_segy_traces(p, tr[:3], 2000)
    assert V.read_velocity_segy(p).x_axis.tolist() == [0, 1, 2]


def test_json_npz_text_round_trips(tmp_path):
    m2, m3 = _ref_models()
    for m in (m2, m3, M.create_constant_velocity(2100.0)):
        V.write_velocity_json(m, tmp_path / "m.json")
        r = V.read_velocity_json(tmp_path / "m.json")
        assert r.velocity_type == m.velocity_type
        assert np.array_equal(np.asarray(r.data, np.float32), np.asarray(m.data, np.float32))
        V.write_velocity_npy(m, tmp_path / "m")
        r = V.read_velocity_npy(tmp_path / "m.npz")
        assert np.array_equal(np.asarray(r.data, np.float32), np.asarray(m.data, np.float32))
        assert V.preview_velocity_file(tmp_path / "m.npz").is_valid
    lin = M.create_linear_gradient_velocity(1500.0, 600.0, 3.0, 0.5)
    V.write_velocity_auto(lin, tmp_path / "lin.txt")
    r = V.read_velocity_auto(tmp_path / "lin.txt")
    assert np.allclose(r.data, lin.data) and np.allclose(r.z_axis, lin.z_axis)
    conv = V.convert_velocity_file(tmp_path / "lin.txt", tmp_path / "lin_int.json")
    assert conv.metadata["velocity_type"] == "interval"
    assert json.load(open(tmp_path / "lin_int.json"))["velocity_type"] == "v_of_z"
    pk = V.create_velocity_from_picks([(1.0, 2000.0), (0.0, 1500.0)], dt=0.25)
    assert pk.data.tolist() == [1500.0, 1625.0, 1750.0, 1875.0, 2000.0]
    assert "Lateral y" in V.get_velocity_summary(m3)


def test_preview_reports_errors_without_raising(tmp_path):
    p = tmp_path / "empty.txt"
    p.write_text("# nothing here\n")
    info = V.preview_velocity_file(p)
    assert not info.is_valid and info.error_message
    assert not V.preview_velocity_file(tmp_path / "missing.txt").is_valid
    with pytest.raises(ValueError):
        V.velocity_info_to_model(info)
