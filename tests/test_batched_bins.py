"""Offset/azimuth binning on the device (here on CPU tensors): the same
classes as the reference's binning table (models/binning.py:136-158), restated
with numpy in this test."""
import numpy as np
import pytest
import torch

from seisproc_b200.batched import OffsetAzimuthBin, bin_indices, offset_azimuth


def _geometry(n=5000, seed=2):
    rs = np.random.RandomState(seed)
    mx, my = rs.uniform(0, 3000, n), rs.uniform(0, 3000, n)
    off, az = rs.uniform(0, 2400, n), rs.uniform(0, 2 * np.pi, n)
    sx, sy = mx - 0.5 * off * np.sin(az), my - 0.5 * off * np.cos(az)
    rx, ry = mx + 0.5 * off * np.sin(az), my + 0.5 * off * np.cos(az)
    return [a.astype(np.float32) for a in (sx, sy, rx, ry)]


def _numpy_classes(g, bins):
    sx, sy, rx, ry = g
    off = np.sqrt((rx - sx) ** 2 + (ry - sy) ** 2).astype(np.float32)
    az = (np.degrees(np.arctan2(rx - sx, ry - sy)) + 360) % 360
    out = []
    for b in bins:
        ok = (off >= b.offset_min) & (off < b.offset_max)
        if b.azimuth_max < b.azimuth_min:
            ok &= (az >= b.azimuth_min) | (az < b.azimuth_max)
        else:
            ok &= (az >= b.azimuth_min) & (az < b.azimuth_max)
        out.append(np.nonzero(ok)[0])
    return out


def _table():
    return [OffsetAzimuthBin(f"o{i}a{j}", 600.0 * i, 600.0 * (i + 1), 90.0 * j, 90.0 * (j + 1))
            for i in range(4) for j in range(4)]


def test_regular_table_matches_numpy():
    g = _geometry()
    bins = _table()
    got = bin_indices(*[torch.from_numpy(a) for a in g], bins)
    want = _numpy_classes(g, bins)
    assert sum(len(w) for w in want) == len(g[0])
    for a, b in zip(got, want):
        assert np.array_equal(a.numpy(), b)


def test_wrapping_and_overlapping_bins():
    g = _geometry(seed=3)
    bins = [OffsetAzimuthBin("north", 0.0, 2500.0, 315.0, 45.0),
            OffsetAzimuthBin("near", 0.0, 800.0),
            OffsetAzimuthBin("off", 0.0, 100.0, enabled=False)]
    got = bin_indices(*[torch.from_numpy(a) for a in g], bins)
    want = _numpy_classes(g, bins[:2])
    assert len(got) == 2
    for a, b in zip(got, want):
        assert np.array_equal(a.numpy(), b)


def test_offset_azimuth_conventions():
    z = torch.zeros(4, dtype=torch.float64)
    rx = torch.tensor([0.0, 10.0, 0.0, -10.0], dtype=torch.float64)
    ry = torch.tensor([10.0, 0.0, -10.0, 0.0], dtype=torch.float64)
    off, az = offset_azimuth(z, z, rx, ry)
    assert torch.allclose(off, torch.full((4,), 10.0))
    assert torch.allclose(az, torch.tensor([0.0, 90.0, 180.0, 270.0], dtype=torch.float64))


def test_invalid_bins_rejected():
    with pytest.raises(ValueError):
        OffsetAzimuthBin("bad", 100.0, 50.0)
    with pytest.raises(ValueError):
        OffsetAzimuthBin("bad", 0.0, 50.0, 0.0, 400.0)


# --- pinned to the reference's own binning (tests/golden/make_binning_golden.py) ---

def _golden_bins(d, table):
    rows = d[f"{table}_bins"]
    return [OffsetAzimuthBin(f"{table}{i}", float(r[0]), float(r[1]), float(r[2]), float(r[3]),
                             enabled=bool(r[4])) for i, r in enumerate(rows)]


def _split(d, key):
    counts = d[key.replace("indices", "counts")]
    return np.split(d[key], np.cumsum(counts)[:-1])


@pytest.mark.parametrize("table", ["ovt", "narrow", "common_offset"])
def test_classes_match_reference_binning_table(table):
    """bin_indices reproduces BinningTable.assign_traces_batch on float32
    geometry, edge traces included, index for index.  Offsets equal the
    reference's bit for bit; azimuths may differ in the last bits (numpy's
    float32 arctan2 is not correctly rounded) without moving any trace across
    a bin edge."""
    from conftest import load_golden
    d = load_golden("binning")
    g = [torch.from_numpy(d[k]) for k in ("source_x", "source_y", "receiver_x", "receiver_y")]
    off, az = offset_azimuth(*g)
    assert np.array_equal(off.numpy(), d["offset"])
    assert float(np.abs(az.numpy() - d["azimuth"]).max()) < 1e-4
    got = bin_indices(*g, _golden_bins(d, table))
    want = _split(d, f"{table}_indices")
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert np.array_equal(np.sort(a.numpy()), b)


def test_closed_intervals_match_reference_get_indices_for_bin():
    """inclusive=True reproduces MigrationGeometry.get_indices_for_bin, whose
    closed intervals put edge traces in both neighbouring bins."""
    from conftest import load_golden
    d = load_golden("binning")
    g = [torch.from_numpy(d[k]) for k in ("source_x", "source_y", "receiver_x", "receiver_y")]
    got = bin_indices(*g, _golden_bins(d, "ovt"), inclusive=True)
    want = _split(d, "ovt_closed_indices")
    assert sum(w.size for w in want) > sum(np.diff(np.r_[0, np.cumsum(d["ovt_counts"])]))
    for a, b in zip(got, want):
        assert np.array_equal(np.sort(a.numpy()), b)
