"""The migrated-cube writer in the reference's layout
(utils/migration_output_storage.py:30-485) and the zarr trace reader
(seisio/gather_readers.py:145-262), on the CPU.  zarr is not installed here:
the array is checked against the zarr format-2 specification (metadata
document, chunk keys, raw little-endian chunks at full chunk size) and read
back by this package's reader; the parquet tables with pandas."""
import json

import numpy as np
import pandas as pd
import pytest

from seisproc_b200.ingest import ZarrDataReader
from seisproc_b200.output_storage import (MigrationOutputStorage, ZarrV2Array,
                                          create_migration_output_storage)


def _cube(nt=37, nil=5, nxl=7, seed=3):
    rs = np.random.RandomState(seed)
    img = rs.randn(nt, nil, nxl).astype(np.float32)
    fold = rs.randint(0, 4, (nt, nil, nxl)).astype(np.float32)
    return img, fold


def test_layout_and_normalised_image(tmp_path):
    img, fold = _cube()
    nt, nil, nxl = img.shape
    st = create_migration_output_storage(tmp_path / "bin0", nt, nil, nxl, dt_ms=2.0, t0_ms=8.0,
                                         d_inline=12.5, d_xline=25.0, inline_start=100,
                                         xline_start=7, x_origin=5.0e5, y_origin=6.0e6,
                                         grid_azimuth_deg=30.0, chunk_size=8)
    for il in range(nil):
        st.write_inline(il, img[:, il, :], fold[:, il, :])
    meta = st.finalize(normalize=True, extra_metadata={"aperture_m": 1000.0})
    out = tmp_path / "bin0"
    # zarr format 2, uncompressed, (n_time, n_traces), inline-major
    za = json.loads((out / "traces.zarr" / ".zarray").read_text())
    assert za["zarr_format"] == 2 and za["compressor"] is None and za["dtype"] == "<f4"
    assert za["shape"] == [nt, nil * nxl] and za["chunks"] == [nt, 8] and za["order"] == "C"
    n_chunks = -(-nil * nxl // 8)
    for j in range(n_chunks):  # every chunk stored at full size
        assert (out / "traces.zarr" / f"0.{j}").stat().st_size == nt * 8 * 4
    got = ZarrV2Array.open(out / "traces.zarr").read()
    f2 = fold.reshape(nt, -1)
    with np.errstate(divide="ignore", invalid="ignore"):
        want = np.where(f2 > 0, img.reshape(nt, -1) / f2, 0.0).astype(np.float32)
    assert np.array_equal(got, want)
    assert np.array_equal(np.load(out / "fold.npy"), f2)
    # headers: the reference's rotated grid coordinates, inline-major
    h = pd.read_parquet(out / "headers.parquet")
    assert list(h.columns) == ["trace_index", "inline", "xline", "cdp_x", "cdp_y",
                               "ensemble_number", "trace_in_ensemble"]
    az = np.radians(30.0)
    il = np.repeat(np.arange(nil), nxl)
    xl = np.tile(np.arange(nxl), nil)
    assert np.array_equal(h["inline"], 100 + il) and np.array_equal(h["xline"], 7 + xl)
    assert np.allclose(h["cdp_x"], 5.0e5 + il * 12.5 * np.sin(az) + xl * 25.0 * np.cos(az))
    assert np.allclose(h["cdp_y"], 6.0e6 + il * 12.5 * np.cos(az) - xl * 25.0 * np.sin(az))
    e = pd.read_parquet(out / "ensemble_index.parquet")
    assert np.array_equal(e["start_trace"], np.arange(nil) * nxl)
    assert np.array_equal(e["end_trace"], np.arange(nil) * nxl + nxl - 1)
    ti = pd.read_parquet(out / "trace_index.parquet")
    assert np.array_equal(ti["global_trace_id"], np.arange(nil * nxl))
    m = json.loads((out / "metadata.json").read_text())
    assert m == json.loads(json.dumps(meta))
    assert m["shape"] == [nt, nil * nxl] and m["n_samples"] == nt and m["sample_rate"] == 2.0
    assert m["migration_info"]["inline_end"] == 100 + nil - 1
    assert m["processing_stats"]["max_fold"] == float(fold.max())
    assert m["migration_params"] == {"aperture_m": 1000.0}


def test_full_cube_without_normalisation_and_reader(tmp_path):
    img, fold = _cube(nt=20, nil=3, nxl=11, seed=5)
    st = MigrationOutputStorage(tmp_path)
    st.initialize_output(n_time=20, n_inline=3, n_xline=11, chunk_size=1000)
    st.write_full_cube(img, fold)
    st.finalize(normalize=False)
    r = ZarrDataReader(tmp_path)  # the directory holding traces.zarr
    assert r.is_transposed and r.shape == (33, 20) and r.get_n_samples() == 20
    flat = img.reshape(20, -1)
    assert np.array_equal(r.read_traces(np.arange(4, 9)), flat[:, 4:9].T)
    sel = np.array([30, 2, 17, 2])
    assert np.array_equal(r.read_traces(sel), flat[:, sel].T)
    with pytest.raises(ValueError):
        st.write_full_cube(img[:, :2], fold[:, :2])


def test_reader_row_major_array_and_refusals(tmp_path):
    a = ZarrV2Array.create(tmp_path / "tr.zarr", (10, 6), (4, 4))
    data = np.arange(60, dtype=np.float32).reshape(10, 6)
    a.write(data)
    r = ZarrDataReader(tmp_path / "tr.zarr")  # no metadata: (n_traces, n_samples)
    assert not r.is_transposed and r.shape == (10, 6)
    assert np.array_equal(r.read_traces(np.array([9, 0, 5])), data[[9, 0, 5]])
    a.write(np.full((10, 3), -1.0, np.float32), col0=2)  # partial chunk rewrite
    assert np.array_equal(ZarrV2Array.open(tmp_path / "tr.zarr").read()[:, 2:5], -np.ones((10, 3)))
    assert np.array_equal(ZarrV2Array.open(tmp_path / "tr.zarr").read()[:, [0, 1, 5]],
                          data[:, [0, 1, 5]])
    meta = json.loads((tmp_path / "tr.zarr" / ".zarray").read_text())
    meta["compressor"] = {"id": "blosc"}
    (tmp_path / "tr.zarr" / ".zarray").write_text(json.dumps(meta))
    with pytest.raises(ValueError, match="compressed"):
        ZarrDataReader(tmp_path / "tr.zarr")
    with pytest.raises(ValueError):
        ZarrDataReader(tmp_path / "nothing")
