"""Opt-in aperture tapers on the GPU: the cosine tapers of the reference's
ApertureController (processors/migration/aperture.py:197-270; its migrators
construct the controller and never apply it) against the FP64 oracle, whose
taper functions are pinned to the controller's own masks."""
import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2
from oracle import pstm_fp64 as O

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4


def _survey(seed, line):
    from seisproc_b200 import synthetic
    return synthetic.survey_3d(n_traces=3000, seed=seed, n_samples=200, extent=1400.0,
                               max_offset=1000.0, n_il=16 if line else 10,
                               n_xl=1 if line else 9, spacing=25.0, n_diffractors=8,
                               aperture=450.0)


def _cols(s):
    il = np.arange(s.n_il)[:, None]
    xl = np.arange(s.n_xl)[None, :]
    return ((s.origin_x + il * s.il_spacing + 0 * xl).ravel(),
            (s.origin_y + 0 * il + xl * s.xl_spacing).ravel())


def _plan(s, **kw):
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    return PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                    origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                    xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                    in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                    max_angle_deg=s.max_angle_deg, **kw)


@pytest.mark.parametrize("line", [False, True])
@pytest.mark.parametrize("forward_only", [False, True])
@pytest.mark.parametrize("tw", [0.1, 0.3])
def test_tapered_plan_matches_fp64_oracle(tw, forward_only, line):
    s = _survey(40 + int(10 * tw) + 2 * line + forward_only, line)
    plan = _plan(s, taper_width=tw, forward_only=forward_only)
    img, fold = plan.migrate(s.traces.cuda(), torch.from_numpy(s.vrms).cuda())
    plan.check()
    plan.close()
    img = img.reshape(s.n_times, -1).cpu().numpy()
    fold = fold.reshape(s.n_times, -1).cpu().numpy()
    cx, cy = _cols(s)
    t_ms = (np.arange(s.n_times, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    args = (s.traces.cpu().numpy(), s.source_x, s.source_y, s.receiver_x, s.receiver_y, cx, cy,
            t_ms, s.vrms.reshape(s.n_times, -1), s.dt_ms, 0.0, s.max_aperture_m,
            s.max_angle_deg)
    oi, of = O.migrate_fp64(*args, taper_width=tw)
    o0, _ = O.migrate_fp64(*args)
    assert rel_l2(img, oi) <= FP32_TOL
    assert np.abs(fold - of).sum() <= max(2, 1e-5 * of.sum())  # fold: the hard masks
    assert rel_l2(oi, o0) > 1e-2  # the tapers change the image


def test_migrator_aperture_taper_matches_oracle():
    """KirchhoffMigrator(aperture_taper=True): offset taper per trace, distance
    and angle tapers per leg, with the migrator's clamp and weight."""
    from seisproc_b200 import models as M
    from seisproc_b200.migrator import KirchhoffMigrator
    d = load_golden("migrator_mini")
    ox, oy, dx, dy, nil, nxl, dt, tmin, v, A, ang, nt, gdt = d["grid"]
    grid = M.OutputGrid(n_time=int(nt), n_inline=int(nil), n_xline=int(nxl), dt=float(gdt),
                        d_inline=float(dx), d_xline=float(dy), t0=0.0, x_origin=float(ox),
                        y_origin=float(oy))
    tw, omin, omax = 0.25, 40.0, 380.0
    cfg = M.MigrationConfig(output_grid=grid, max_aperture_m=float(A), max_angle_deg=float(ang),
                            min_offset_m=omin, max_offset_m=omax, taper_width=tw)
    mig = KirchhoffMigrator(M.create_constant_velocity(float(v)), cfg, use_traveltime_lut=False,
                            aperture_taper=True)
    gather = M.SeismicData(traces=d["traces"], sample_rate=float(dt))
    geom = M.MigrationGeometry(d["source_x"], d["source_y"], d["receiver_x"], d["receiver_y"])
    img, fold = mig.migrate_gather(gather, geom)
    off = geom.offset
    sel = np.nonzero((off >= omin) & (off <= omax))[0]
    w = O.offset_taper_fp64(off[sel], omin, omax, tw)
    tr = d["traces"][:, sel].astype(np.float64) * w[None, :]
    il = np.arange(int(nil))[:, None]
    xl = np.arange(int(nxl))[None, :]
    cx = (ox + il * dx + 0 * xl).ravel()
    cy = (oy + 0 * il + xl * dy).ravel()
    t_ms = np.arange(int(nt)) * float(gdt) * 1000.0
    oi, of = O.migrate_fp64(tr, geom.source_x[sel], geom.source_y[sel], geom.receiver_x[sel],
                            geom.receiver_y[sel], cx, cy, t_ms, float(v), float(dt), 0.0,
                            float(A), float(ang), weight="spreading", clamp="migrator",
                            taper_width=tw)
    assert rel_l2(img.reshape(int(nt), -1).cpu().numpy(), oi) <= FP32_TOL
    assert np.abs(fold.reshape(int(nt), -1).cpu().numpy() - of).sum() <= 2
    plain = KirchhoffMigrator(M.create_constant_velocity(float(v)), cfg,
                              use_traveltime_lut=False)
    p_img, _ = plain.migrate_gather(gather, geom)
    assert rel_l2(img.cpu().numpy(), p_img.cpu().numpy()) > 1e-2  # default: no taper


def test_tapered_plan_refusals():
    from seisproc_b200.batched import BatchedPSTM
    s = _survey(60, False)
    plan = _plan(s, taper_width=0.2)
    v = torch.from_numpy(s.vrms).cuda()
    img, _ = plan.migrate(s.traces.cuda(), v)
    with pytest.raises(Exception, match="taper"):
        plan.demigrate(img, v)
    with pytest.raises(Exception, match="taper"):
        plan.velocity_gradient(img, v)
    with pytest.raises(Exception, match="taper"):
        BatchedPSTM([plan], v)
    plan.check()
    plan.close()
    with pytest.raises(Exception, match="taper"):
        _plan(s, taper_width=0.2, storage="bf16")
    with pytest.raises(Exception, match="taper"):
        _plan(s, taper_width=0.2, variant=1)
    with pytest.raises(ValueError, match="taper_width"):
        _plan(s, taper_width=1.5)
