"""Batched persistent launch over offset/azimuth classes, CUDA-graph replay,
and the shape autotuner, on the GPU."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _classes(storage="f32", forward_only=False):
    from seisproc_b200 import synthetic
    from seisproc_b200.kirchhoff import PSTMPlan
    surveys = synthetic.survey_classes([900, 300, 1500, 50], seed=3, n_offset_bins=2,
                                       n_azimuth_bins=2, max_offset=1200.0, n_samples=200,
                                       extent=1000.0, n_il=10, n_xl=9, spacing=25.0,
                                       n_diffractors=6, aperture=400.0)
    dev = torch.device("cuda")
    plans = []
    for s in surveys:
        c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
             for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
        plans.append(PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times,
                              origin_x=s.origin_x, origin_y=s.origin_y, il_dx=s.il_spacing,
                              il_dy=0.0, xl_dx=0.0, xl_dy=s.xl_spacing, t0_ms=0.0,
                              dt_ms=s.dt_ms, n_samples=s.n_samples, in_t0_ms=0.0,
                              in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                              max_angle_deg=s.max_angle_deg, storage=storage,
                              forward_only=forward_only))
    v = torch.from_numpy(surveys[0].vrms).to(dev)
    return surveys, plans, v


@pytest.mark.parametrize("storage,forward_only", [("f32", False), ("f32", True), ("bf16", False),
                                                  ("bf16", True)])
def test_batched_matches_per_class_plans(storage, forward_only):
    """Forward_only float32 class plans run the batched kernel over
    intercept-form rows, the others over (x, dx) or 16-bit rows."""
    from seisproc_b200.batched import BatchedPSTM
    surveys, plans, v = _classes(storage, forward_only)
    traces = [s.traces.cuda() for s in surveys]
    b = BatchedPSTM(plans, v)
    b.load(traces)
    b.migrate()
    b.check()
    for p, s, img, fold in zip(plans, surveys, b.images, b.folds):
        ri, rf = p.migrate(s.traces.cuda(), v)
        p.check()
        assert torch.equal(img, ri), "batched image differs from the per-class launch"
        assert torch.equal(fold, rf)
    b.close()


def test_batched_graph_replay_follows_inputs():
    from seisproc_b200.batched import BatchedPSTM
    surveys, plans, v = _classes()
    bufs = [s.traces.cuda().clone() for s in surveys]
    b = BatchedPSTM(plans, v, with_fold=False)
    b.capture(bufs)
    ref0 = [t.clone() for t in b.images]
    for t in bufs:
        t.mul_(-2.0)
    b.replay()
    torch.cuda.synchronize()
    b.check()
    for r, img in zip(ref0, b.images):
        assert rel_l2(img.cpu().numpy(), -2.0 * r.cpu().numpy()) <= 1e-6
    b.close()


def test_autotuner_picks_and_caches(tmp_path, monkeypatch):
    from seisproc_b200 import autotune
    monkeypatch.setenv("SEISPSTM_TUNE_CACHE", str(tmp_path / "tune.json"))
    surveys, plans, v = _classes()
    s = surveys[2]
    p0 = plans[2]
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]

    def make(var):
        return PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                        origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                        xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                        in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                        max_angle_deg=s.max_angle_deg, variant=var)
    key = autotune.problem_key(s.n_xl, s.n_times, s.n_samples, 1500 / 90, "f32")
    best, times = autotune.tune(make, s.traces.cuda(), v, key, autotune.candidates(s.n_xl))
    assert best in autotune.GRID_SHAPES and set(times) == set(autotune.GRID_SHAPES)
    assert autotune.cached_variant(key) == best
    best2, times2 = autotune.tune(make, s.traces.cuda(), v, key, autotune.candidates(s.n_xl))
    assert best2 == best and times2 == {}


def test_from_survey_matches_per_class_plans():
    """A whole survey binned on the device into offset/azimuth classes, one
    batched launch: each class image equals a plan built from that class's
    traces selected on the host."""
    from seisproc_b200 import synthetic
    from seisproc_b200.batched import BatchedPSTM, OffsetAzimuthBin
    from seisproc_b200.kirchhoff import PSTMPlan
    s = synthetic.survey_3d(n_traces=4000, seed=12, n_samples=200, extent=1000.0,
                            max_offset=1200.0, n_il=10, n_xl=9, spacing=25.0, n_diffractors=6,
                            aperture=400.0)
    dev = torch.device("cuda")
    bins = [OffsetAzimuthBin(f"o{i}a{j}", 400.0 * i, 400.0 * (i + 1), 180.0 * j, 180.0 * (j + 1))
            for i in range(3) for j in range(2)]
    kw = dict(n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
              origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0, xl_dy=s.xl_spacing,
              t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples, in_t0_ms=0.0, in_dt_ms=s.dt_ms,
              max_aperture_m=s.max_aperture_m, max_angle_deg=s.max_angle_deg)
    coords = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
              for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    v = torch.from_numpy(s.vrms).to(dev)
    tr = s.traces.to(dev)
    b = BatchedPSTM.from_survey(tr, *coords, bins, v, **kw)
    b.migrate()
    b.check()
    off = np.sqrt((s.receiver_x - s.source_x) ** 2 + (s.receiver_y - s.source_y) ** 2)
    az = (np.degrees(np.arctan2(s.receiver_x - s.source_x, s.receiver_y - s.source_y)) + 360) % 360
    assert sum(int(i.numel()) for i in b.indices) == s.n_traces
    for bn, idx, img, fold in zip(b.bins, b.indices, b.images, b.folds):
        sel = np.nonzero((off >= bn.offset_min) & (off < bn.offset_max) &
                         (az >= bn.azimuth_min) & (az < bn.azimuth_max))[0]
        assert np.array_equal(idx.cpu().numpy(), sel)
        c = [a[torch.from_numpy(sel).to(dev)] for a in coords]
        p = PSTMPlan(*c, **kw)
        ri, rf = p.migrate(tr[:, torch.from_numpy(sel).to(dev)], v)
        p.check()
        assert torch.equal(img, ri) and torch.equal(fold, rf)
        p.close()
    b.close()


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_engine_migrate_bins_full_matches_per_bin_calls(storage):
    """MigrationEngine.migrate_bins_full (the bins in pipelined groups of
    batched launches: one bin per group, then every bin in one group) gives
    each bin the image and fold that migrate_bin_full gives it alone, into new
    arrays or into the caller's page-locked buffers."""
    from seisproc_b200.engine import MigrationEngine
    surveys, plans, v = _classes(storage)
    for p in plans:
        p.close()
    s0 = surveys[0]
    kw = dict(origin_x=s0.origin_x, origin_y=s0.origin_y, il_spacing=s0.il_spacing,
              xl_spacing=s0.xl_spacing, azimuth_deg=0.0, n_il=s0.n_il, n_xl=s0.n_xl,
              dt_ms=s0.dt_ms, t_min_ms=0.0, n_times=s0.n_times,
              max_aperture_m=s0.max_aperture_m, max_angle_deg=s0.max_angle_deg,
              velocity_model=s0.vrms)
    eng = MigrationEngine(storage=storage)
    bins = [{"traces": s.traces.cpu().numpy(), "source_x": s.source_x, "source_y": s.source_y,
             "receiver_x": s.receiver_x, "receiver_y": s.receiver_y} for s in surveys]
    res = eng.migrate_bins_full(bins, **kw)
    shape = (s0.n_times, s0.n_il, s0.n_xl)
    outs = [(torch.empty(shape, pin_memory=True), torch.empty(shape, pin_memory=True))
            for _ in bins]
    eng.batch_groups = 1
    res2 = eng.migrate_bins_full(bins, out=outs, **kw)
    for b, (img, fold), (img2, fold2) in zip(bins, res, res2):
        ri, rf = eng.migrate_bin_full(b["traces"], b["source_x"], b["source_y"],
                                      b["receiver_x"], b["receiver_y"], **kw)
        assert img.shape == ri.shape and fold.shape == rf.shape
        assert rel_l2(img, ri) <= 1e-6 and np.array_equal(fold, rf)
        assert np.array_equal(img2.numpy(), img) and np.array_equal(fold2.numpy(), fold)


def test_autotuner_choice_is_used_and_cached(tmp_path, monkeypatch):
    """choose_variant times the candidate shapes (256- and 128-sample windows
    among them) on a crop, caches the winner under the device and library
    ABI, and the engine builds its plans with that shape; a second choice is a
    cache hit that times nothing."""
    import json
    from seisproc_b200 import autotune
    from seisproc_b200.engine import MigrationEngine
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("SEISPSTM_TUNE_CACHE", str(cache))
    surveys, plans, v = _classes()
    for p in plans:
        p.close()
    s = surveys[2]
    dev = torch.device("cuda")
    coords = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
              for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    kw = dict(n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
              origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0, xl_dy=s.xl_spacing,
              t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples, in_t0_ms=0.0, in_dt_ms=s.dt_ms,
              max_aperture_m=s.max_aperture_m, max_angle_deg=s.max_angle_deg, forward_only=True)
    best = autotune.choose_variant(coords, velocity=v, **kw)
    d = json.loads(cache.read_text())
    (tag, entries), = d.items()
    assert tag == autotune.device_tag()
    (key, entry), = entries.items()
    assert entry["variant"] == best and set(map(int, entry["ms"])) == set(autotune.GRID_SHAPES)
    assert {10, 11} <= set(autotune.GRID_SHAPES)
    mtime = cache.stat().st_mtime_ns
    assert autotune.choose_variant(coords, velocity=v, **kw) == best
    assert cache.stat().st_mtime_ns == mtime  # a hit writes nothing
    eng = MigrationEngine()
    eng.migrate_bin_full(s.traces.cpu().numpy(), s.source_x, s.source_y, s.receiver_x,
                         s.receiver_y, s.origin_x, s.origin_y, s.il_spacing, s.xl_spacing, 0.0,
                         s.n_il, s.n_xl, s.dt_ms, 0.0, s.n_times, max_aperture_m=s.max_aperture_m,
                         max_angle_deg=s.max_angle_deg, velocity_model=s.vrms)
    assert eng.last_stats["variant"] == best


@pytest.mark.parametrize("shape", [10, 11])
def test_short_window_shapes_match_default_shape(shape):
    """The 256- and 128-sample windows give the fold of the 512-sample shape
    exactly and its image to float rounding: each window stages its rows from
    its own first sample, and that offset enters the float32 sample index, so
    the fractional parts round differently (measured 2.4e-6)."""
    surveys, plans, v = _classes()
    from seisproc_b200.kirchhoff import PSTMPlan
    s = surveys[2]
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    kw = dict(n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
              origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0, xl_dy=s.xl_spacing,
              t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples, in_t0_ms=0.0, in_dt_ms=s.dt_ms,
              max_aperture_m=s.max_aperture_m, max_angle_deg=s.max_angle_deg)
    ref = PSTMPlan(*c, variant=3, **kw)
    alt = PSTMPlan(*c, variant=shape, **kw)
    ri, rf = ref.migrate(s.traces.cuda(), v)
    ai, af = alt.migrate(s.traces.cuda(), v)
    ref.check()
    alt.check()
    assert alt.stats()["t_window"] == {10: 256, 11: 128}[shape]
    assert torch.equal(af, rf)
    assert rel_l2(ai.cpu().numpy(), ri.cpu().numpy()) <= 1e-5
    for p in plans + [ref, alt]:
        p.close()


def test_batched_fold_with_a_long_tile_list():
    """A batch where one class's tile list holds 70 000 traces takes the 32-bit
    fold histogram for every class (one shared-memory layout per launch); the
    folds and images equal the per-class launches, which choose their
    histograms alone (16-bit for the small class)."""
    from seisproc_b200.batched import BatchedPSTM
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    n_s = n_t = 64
    rs = np.random.RandomState(70)
    plans, traces = [], []
    for n in (70000, 500):
        # every trace near one point between the 2 x 2 columns
        c = [torch.from_numpy(1012.5 + rs.uniform(-5.0, 5.0, n)).to(dev) for _ in range(4)]
        plans.append(PSTMPlan(*c, n_il=2, n_xl=2, n_times=n_t, origin_x=1000.0,
                              origin_y=1000.0, il_dx=25.0, il_dy=0.0, xl_dx=0.0, xl_dy=25.0,
                              t0_ms=0.0, dt_ms=4.0, n_samples=n_s, in_t0_ms=0.0, in_dt_ms=4.0,
                              max_aperture_m=500.0, max_angle_deg=60.0, forward_only=True,
                              variant=1))
        traces.append(torch.from_numpy(rs.standard_normal((n_s, n)).astype(np.float32)).to(dev))
    assert plans[0].stats()["list_entries"] == 70000
    v = torch.full((n_t,), 2000.0, device=dev)
    b = BatchedPSTM(plans, v)
    b.load(traces)
    b.migrate()
    b.check()
    for p, tr, img, fold in zip(plans, traces, b.images, b.folds):
        ri, rf = p.migrate(tr, v)
        p.check()
        assert torch.equal(fold, rf)
        assert torch.equal(img, ri)
    assert float(b.folds[0].max()) == 70000.0
    b.close()
    for p in plans:
        p.close()
