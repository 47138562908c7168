"""Inline slabs of the multi-GPU path on one GPU, slab after slab: the slabs'
images put side by side equal the one-plan image, and the slabs' demigration
partials add up to the one-plan demigration."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _survey():
    from seisproc_b200 import synthetic
    return synthetic.survey_3d(n_traces=3000, seed=41, n_samples=200, extent=1200.0,
                               max_offset=800.0, n_il=9, n_xl=6, spacing=25.0, n_diffractors=6,
                               aperture=400.0, utm_origin=(5.0e5, 6.0e6))


def _kw(s):
    return dict(n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                max_angle_deg=s.max_angle_deg)


@pytest.mark.parametrize("world", [2, 3])
def test_slabs_match_one_plan(world):
    from seisproc_b200.kirchhoff import PSTMPlan
    from seisproc_b200.sharding import ShardedPSTM
    s = _survey()
    dev = torch.device("cuda")
    vel = torch.from_numpy(s.vrms).to(dev).reshape(s.n_times, s.n_il, s.n_xl)
    coords = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
              for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan = PSTMPlan(*coords, **_kw(s))
    tr = s.traces.to(dev)
    full_img, full_fold = plan.migrate(tr, vel)
    m = torch.randn((s.n_times, s.n_il, s.n_xl), device=dev,
                    generator=torch.Generator(device=dev).manual_seed(3))
    full_d = plan.demigrate(m, vel)
    plan.check()
    imgs, folds, dsum = [], [], torch.zeros_like(full_d)
    for r in range(world):
        sh = ShardedPSTM(s.source_x, s.source_y, s.receiver_x, s.receiver_y, velocity=vel,
                         rank=r, world=world, **_kw(s))
        assert sh.halo.size < s.n_traces
        img, fold = sh.migrate(tr)
        imgs.append(img)
        folds.append(fold)
        dsum += sh.demigrate_partial(m[:, sh.il0:sh.il1].contiguous())
        sh.plan.check()
        sh.close()
    img = torch.cat(imgs, 1)
    fold = torch.cat(folds, 1)
    assert rel_l2(img.cpu().numpy(), full_img.cpu().numpy()) <= 1e-5
    assert torch.equal(fold, full_fold)
    assert rel_l2(dsum.cpu().numpy(), full_d.cpu().numpy()) <= 1e-5
    plan.close()


def test_one_rank_cgls_reduces_misfit():
    from seisproc_b200.sharding import ShardedPSTM
    s = _survey()
    dev = torch.device("cuda")
    vel = torch.from_numpy(s.vrms).to(dev).reshape(s.n_times, s.n_il, s.n_xl)
    sh = ShardedPSTM(s.source_x, s.source_y, s.receiver_x, s.receiver_y, velocity=vel, **_kw(s))
    d = sh.demigrate(torch.randn((s.n_times, s.n_il, s.n_xl), device=dev,
                                 generator=torch.Generator(device=dev).manual_seed(9)))
    m, hist = sh.cgls(d, n_iter=5)
    assert m.shape == (s.n_times, s.n_il, s.n_xl)
    assert hist[-1][1] < 0.7
    sh.close()
