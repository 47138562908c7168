"""Trace readers on the host: the reference's NumpyDataReader interface and a
memory-mapped SEG-Y reader (IEEE and IBM samples) against the file writer."""
import numpy as np
import pytest

from seisproc_b200 import ingest as I
from seisproc_b200 import velocity_io as V


def test_numpy_reader_matches_reference_interface():
    d = np.random.RandomState(1).standard_normal((50, 37)).astype(np.float32)
    r = I.NumpyDataReader(d)
    assert r.get_n_samples() == 37 and r.n_traces == 50
    idx = np.array([4, 9, 9, 0, 49])
    assert np.array_equal(r.read_traces(idx), d[idx])


@pytest.mark.parametrize("fmt", [1, 5])
def test_segy_reader_memory_map(tmp_path, fmt):
    rs = np.random.RandomState(2)
    tr = rs.uniform(-3, 3, (300, 123)).astype(np.float32)
    p = tmp_path / "t.sgy"
    V.write_segy_traces(p, tr, 4000, cdp=np.arange(300), fmt=fmt)
    r = I.SegyDataReader(p)
    assert r.n_traces == 300 and r.get_n_samples() == 123
    idx = np.array([299, 0, 17, 17, 150])
    got = r.read_traces(idx)
    assert got.dtype == np.float32 and got.shape == (5, 123)
    tol = 0 if fmt == 5 else 2.0 ** -20
    assert np.all(np.abs(got - tr[idx]) <= tol * np.abs(tr[idx]))
    assert np.array_equal(got, V.read_segy_traces(p)["traces"][idx])


def test_segy_reader_rejects_integer_samples(tmp_path):
    p = tmp_path / "i.sgy"
    V.write_segy_traces(p, np.zeros((2, 10), np.float32), 4000, fmt=5)
    raw = bytearray(p.read_bytes())
    raw[3224:3226] = (3).to_bytes(2, "big")  # int16 samples
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError):
        I.SegyDataReader(p)
