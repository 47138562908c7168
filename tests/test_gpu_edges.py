"""Edge shapes on the GPU against the FP64 oracle: one trace and one output
sample, trace counts and grids that fill no warp or tile, output windows and
trace lengths that are not multiples of the kernel's, outputs longer than the
input traces, and traces too long for the staged kernel."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import pstm_fp64 as O

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4          # rel-L2 of the image against the FP64 oracle
FOLD_FLIP_FRAC = 1e-5    # fold pairs that may flip at a float32 mask boundary

SHAPES = [  # traces, inlines, crosslines, input samples, output samples
    (1, 1, 1, 50, 1),
    (1, 1, 1, 60, 60),
    (33, 5, 7, 37, 37),
    (300, 9, 3, 513, 513),
    (64, 2, 1, 80, 600),
    (500, 17, 1, 129, 129),
]


def _survey(n_tr, n_il, n_xl, n_s, n_t, seed):
    from seisproc_b200 import synthetic
    return synthetic.survey_3d(n_traces=n_tr, seed=seed, n_samples=n_s, n_times=n_t,
                               extent=max(n_il, n_xl) * 25.0 + 200.0, max_offset=400.0,
                               n_il=n_il, n_xl=n_xl, spacing=25.0, n_diffractors=3,
                               aperture=300.0)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("forward_only", [False, True])
def test_edge_shapes_match_fp64_oracle(shape, forward_only):
    from seisproc_b200.kirchhoff import PSTMPlan
    n_tr, n_il, n_xl, n_s, n_t = shape
    s = _survey(*shape, seed=sum(shape))
    # white-noise traces: every contributing pair shows in the image
    tr = torch.from_numpy(np.random.RandomState(sum(shape)).standard_normal((n_s, n_tr))
                          .astype(np.float32))
    vrms = s.vrms
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan = PSTMPlan(*c, n_il=n_il, n_xl=n_xl, n_times=n_t, origin_x=s.origin_x,
                    origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                    xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=n_s, in_t0_ms=0.0,
                    in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                    max_angle_deg=s.max_angle_deg, forward_only=forward_only)
    img, fold = plan.migrate(tr.to(dev), torch.from_numpy(vrms).to(dev))
    plan.check()
    plan.close()
    img = img.reshape(n_t, -1).cpu().numpy()
    fold = fold.reshape(n_t, -1).cpu().numpy()
    il = np.arange(n_il)[:, None]
    xl = np.arange(n_xl)[None, :]
    cx = (s.origin_x + il * s.il_spacing + 0 * xl).ravel()
    cy = (s.origin_y + 0 * il + xl * s.xl_spacing).ravel()
    t_ms = (np.arange(n_t, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    oi, of = O.migrate_fp64(tr.numpy(), s.source_x, s.source_y, s.receiver_x,
                            s.receiver_y, cx, cy, t_ms, vrms.reshape(n_t, -1), s.dt_ms, 0.0,
                            s.max_aperture_m, s.max_angle_deg)
    assert np.isfinite(img).all()
    assert np.abs(fold - of).sum() <= max(2, FOLD_FLIP_FRAC * of.sum())
    if of.sum() == 0:
        assert np.abs(img).max() == 0
    else:
        assert rel_l2(img, oi) <= FP32_TOL


def test_traces_too_long_for_the_staged_kernel():
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    c = [torch.zeros(8, device=dev) for _ in range(4)]
    with pytest.raises(ValueError, match="too long"):
        PSTMPlan(*c, n_il=4, n_xl=4, n_times=100, origin_x=0.0, origin_y=0.0, il_dx=25.0,
                 il_dy=0.0, xl_dx=0.0, xl_dy=25.0, t0_ms=0.0, dt_ms=4.0, n_samples=60000,
                 in_t0_ms=0.0, in_dt_ms=4.0, max_aperture_m=500.0, max_angle_deg=60.0)


@pytest.mark.parametrize("variant", [1, 3])
@pytest.mark.parametrize("n_tr", [65535, 65536])
def test_fold_counts_of_a_full_tile_list(n_tr, variant):
    """Every trace at one point, so one tile list holds all of them and each
    column's fold histogram takes n_tr counts in one bin: 65535 traces use the
    16-bit counts, 65536 the 32-bit histogram; the fold is exact either way."""
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    n_s = n_t = 64
    # the point sits between the 2 x 2 columns, 17.7 m from each: with
    # V = 2000 m/s and dt = 4 ms, z = 4 k m, so tan(60) z exceeds 17.7 m from
    # sample 3 on (13.9 m at sample 2, 20.8 m at sample 3)
    p = np.full(n_tr, 1012.5)
    c = [torch.from_numpy(p.copy()).to(dev) for _ in range(4)]
    plan = PSTMPlan(*c, n_il=2, n_xl=2, n_times=n_t, origin_x=1000.0, origin_y=1000.0,
                    il_dx=25.0, il_dy=0.0, xl_dx=0.0, xl_dy=25.0, t0_ms=0.0, dt_ms=4.0,
                    n_samples=n_s, in_t0_ms=0.0, in_dt_ms=4.0, max_aperture_m=500.0,
                    max_angle_deg=60.0, forward_only=True, variant=variant)
    assert plan.stats()["list_entries"] == n_tr
    tr = torch.from_numpy(np.random.RandomState(n_tr).standard_normal((n_s, n_tr))
                          .astype(np.float32)).to(dev)
    img, fold = plan.migrate(tr, torch.full((n_t,), 2000.0, device=dev))
    plan.check()
    plan.close()
    fold = fold.reshape(n_t, -1).cpu().numpy()
    assert (fold[:3] == 0).all() and (fold[3:] == n_tr).all()
    assert torch.isfinite(img).all()
