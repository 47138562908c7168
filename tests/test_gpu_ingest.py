"""Streaming a reader's traces into the engine on the GPU: the same image as the
transposed-array path, with chunks that do not divide the trace count."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _survey():
    from seisproc_b200 import synthetic
    return synthetic.survey_3d(n_traces=5000, seed=44, n_samples=180, extent=1200.0,
                               max_offset=900.0, n_il=8, n_xl=7, spacing=25.0, n_diffractors=6,
                               aperture=400.0)


def _kw(s):
    return dict(origin_x=s.origin_x, origin_y=s.origin_y, il_spacing=s.il_spacing,
                xl_spacing=s.xl_spacing, azimuth_deg=0.0, n_il=s.n_il, n_xl=s.n_xl,
                dt_ms=s.dt_ms, t_min_ms=0.0, n_times=s.n_times, max_aperture_m=s.max_aperture_m,
                max_angle_deg=s.max_angle_deg, normalize=True, velocity_model=s.vrms)


@pytest.mark.parametrize("blocks", [1, 3])
@pytest.mark.parametrize("kind", ["numpy", "segy", "zarr"])
def test_reader_path_equals_array_path(tmp_path, kind, blocks):
    from seisproc_b200 import ingest as I
    from seisproc_b200 import velocity_io as V
    from seisproc_b200.engine import MigrationEngine
    s = _survey()
    tr_major = np.ascontiguousarray(s.traces.cpu().numpy().T)  # (n_traces, n_samples)
    if kind == "numpy":
        reader = I.NumpyDataReader(tr_major)
    elif kind == "segy":
        p = tmp_path / "bin.sgy"
        V.write_segy_traces(p, tr_major, int(s.dt_ms * 1000), fmt=5)
        reader = I.SegyDataReader(p)
    else:
        # the reference import's layout: (n_samples, n_traces) beside metadata.json
        import json
        from seisproc_b200.output_storage import ZarrV2Array
        ZarrV2Array.create(tmp_path / "traces.zarr", tr_major.T.shape, (s.n_samples, 1000)
                           ).write(np.ascontiguousarray(tr_major.T))
        (tmp_path / "metadata.json").write_text(json.dumps(
            {"n_samples": s.n_samples, "n_traces": s.n_traces}))
        reader = I.ZarrDataReader(tmp_path)
        assert reader.is_transposed
    rs = np.random.RandomState(3)
    idx = np.sort(rs.choice(s.n_traces, 3700, replace=False))  # one bin's traces
    coords = [np.asarray(a)[idx] for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    eng = MigrationEngine()
    if blocks > 1:
        eng.block_traces = idx.size // blocks  # both paths split the bin the same way
    img_r, fold_r = eng.migrate_bin_from_reader(reader, idx, *coords, chunk_traces=1000,
                                                reader_threads=3, **_kw(s))
    assert eng.last_stats["blocks"] == blocks
    img_a, fold_a = eng.migrate_bin_full(reader.read_traces(idx).T, *coords, **_kw(s))
    assert np.array_equal(fold_r, fold_a)
    assert np.array_equal(img_r, img_a)
    assert np.abs(img_a).max() > 0


def test_block_pipelined_upload_matches_single_plan():
    """A bin split into blocks of traces (one plan each, uploads pipelined
    against the migrations, partial images summed) gives the single-plan image
    to float rounding and the same fold."""
    from seisproc_b200.engine import MigrationEngine
    s = _survey()
    tr = s.traces.cpu().numpy()
    host = torch.empty(tr.shape, dtype=torch.float32, pin_memory=True)
    host.copy_(torch.from_numpy(tr))
    coords = (s.source_x, s.source_y, s.receiver_x, s.receiver_y)
    eng = MigrationEngine()
    one, f1 = eng.migrate_bin_full(host.numpy(), *coords, **_kw(s))
    assert eng.last_stats["blocks"] == 1
    eng.block_traces = 1200  # 5000 traces -> 4 blocks
    four, f4 = eng.migrate_bin_full(host.numpy(), *coords, **_kw(s))
    assert eng.last_stats["blocks"] == 4
    four_pageable, _ = eng.migrate_bin_full(tr, *coords, **_kw(s))
    assert np.array_equal(f1, f4)
    assert np.linalg.norm(four - one) <= 1e-6 * np.linalg.norm(one)
    assert np.array_equal(four, four_pageable)
