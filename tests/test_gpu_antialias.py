"""Causal-integrated triangle anti-alias filter on the GPU against the FP64
oracle (the reference has no anti-alias implementation on its migration path;
processors/migration/antialias.py:48-366 is never called by a migrator)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import pstm_fp64 as O

pytestmark = pytest.mark.gpu


def _survey(seed=31, noise=0.03, f_peak=30.0):
    from seisproc_b200 import synthetic
    return synthetic.survey_3d(n_traces=500, seed=seed, n_samples=160, extent=700.0,
                               max_offset=500.0, n_il=6, n_xl=5, spacing=25.0, n_diffractors=5,
                               aperture=350.0, noise_rel=noise, f_peak=f_peak)


def _cols(s):
    il = np.arange(s.n_il)[:, None]
    xl = np.arange(s.n_xl)[None, :]
    return ((s.origin_x + il * s.il_spacing + 0 * xl).ravel(),
            (s.origin_y + 0 * il + xl * s.xl_spacing).ravel())


def _gpu(s, storage="f32", aa=True, aa_dx=None, aa_dy=None, lmax=16.0):
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan = PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                    origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                    xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                    in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                    max_angle_deg=s.max_angle_deg, storage=storage, antialias=aa,
                    aa_dx=s.il_spacing if aa_dx is None else aa_dx,
                    aa_dy=s.xl_spacing if aa_dy is None else aa_dy, aa_max_halfwidth=lmax)
    img, fold = plan.migrate(s.traces.cuda(), torch.from_numpy(s.vrms).cuda())
    plan.check()
    plan.close()
    return img.reshape(s.n_times, -1).cpu().numpy(), fold.reshape(s.n_times, -1).cpu().numpy()


def _oracle(s, lmax=16.0):
    cx, cy = _cols(s)
    t_ms = (np.arange(s.n_times, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    return O.migrate_fp64(s.traces.cpu().numpy(), s.source_x, s.source_y, s.receiver_x,
                          s.receiver_y, cx, cy, t_ms, s.vrms.reshape(s.n_times, -1), s.dt_ms, 0.0,
                          s.max_aperture_m, s.max_angle_deg, antialias=True, dx_out=s.il_spacing,
                          dy_out=s.xl_spacing, l_max=lmax)


def test_antialias_matches_fp64_oracle():
    s = _survey()
    img, fold = _gpu(s)
    oi, of = _oracle(s)
    assert rel_l2(img, oi) <= 1e-4
    assert np.abs(fold - of).sum() <= 2


def test_unit_halfwidth_reduces_to_plain_interpolation():
    """With zero bin spacing the triangle half-width clamps to 1 sample, where
    the filter is the identity: the result equals the plain kernel's."""
    s = _survey(seed=32)
    a, _ = _gpu(s, aa=True, aa_dx=0.0, aa_dy=0.0)
    b, _ = _gpu(s, aa=False)
    assert rel_l2(a, b) <= 1e-4


def test_antialias_attenuates_steep_dips():
    """The filter can only smooth: the anti-aliased image has less energy than
    the unfiltered one on noisy data."""
    s = _survey(seed=33, noise=0.3)
    a, _ = _gpu(s, aa=True)
    b, _ = _gpu(s, aa=False)
    assert np.linalg.norm(a) < np.linalg.norm(b)


@pytest.mark.parametrize("storage,tol", [("f16", 1e-3), ("bf16", 5e-3)])
def test_antialias_16bit_inputs_error_vs_fp64(storage, tol):
    s = _survey(seed=34)
    img, _ = _gpu(s, storage=storage)
    oi, _ = _oracle(s)
    assert rel_l2(img, oi) <= tol
