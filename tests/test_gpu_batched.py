"""Batched persistent launch over offset/azimuth classes, CUDA-graph replay,
and the shape autotuner, on the GPU."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _classes(storage="f32"):
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
                              max_angle_deg=s.max_angle_deg, storage=storage))
    v = torch.from_numpy(surveys[0].vrms).to(dev)
    return surveys, plans, v


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_batched_matches_per_class_plans(storage):
    from seisproc_b200.batched import BatchedPSTM
    surveys, plans, v = _classes(storage)
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
    monkeypatch.setattr(autotune, "_CACHE_PATH", str(tmp_path / "tune.json"))
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
