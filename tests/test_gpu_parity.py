"""GPU parity of the sm_100a PSTM kernels against the reference's own outputs
(golden fixtures made by running it) and against the FP64 oracle.

Tolerances: FP32 image within 1e-4 relative L2 of the reference (the target
for plain FP32); fold equal to the reference's except for pairs that sit
within float32 rounding of a mask boundary (at most 1e-5 of all pairs).
"""
import numpy as np
import pytest
import torch

from conftest import golden_grid, load_golden, rel_l2
from oracle import pstm_fp64 as O

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4
FOLD_FLIP_FRAC = 1e-5


def _engine():
    from seisproc_b200.engine import MigrationEngine
    return MigrationEngine()


def _run_golden(name):
    d = load_golden(name)
    g = golden_grid(d)
    nt = int(d["n_times"])
    img, fold = _engine().migrate_bin_full(
        traces=d["traces"], source_x=d["source_x"], source_y=d["source_y"],
        receiver_x=d["receiver_x"], receiver_y=d["receiver_y"], origin_x=g["origin_x"],
        origin_y=g["origin_y"], il_spacing=g["il_spacing"], xl_spacing=g["xl_spacing"],
        azimuth_deg=0.0, n_il=g["n_il"], n_xl=g["n_xl"], dt_ms=g["dt_ms"],
        t_min_ms=g["t_min_ms"], n_times=nt, velocity_mps=g["velocity_mps"],
        max_aperture_m=g["max_aperture_m"], max_angle_deg=g["max_angle_deg"], normalize=False,
        use_time_dependent_aperture=bool(d["tda"]))
    return d, img, fold


@pytest.mark.parametrize("name", ["full_2d_small", "full_2d_tda_tmin", "full_3d_mini"])
def test_engine_matches_reference_golden(name):
    d, img, fold = _run_golden(name)
    assert img.shape == d["image"].shape
    err = rel_l2(img, d["image"])
    flips = np.abs(fold - d["fold"]).sum()
    assert err <= FP32_TOL, f"{name}: rel-L2 {err:.3e}"
    assert flips <= max(2, FOLD_FLIP_FRAC * d["fold"].sum()), f"{name}: {flips} fold flips"


def test_full_2d_config_matches_reference():
    """The full-size 2D workload (2880 traces x 501 samples -> 240 x 501)."""
    import hashlib
    from seisproc_b200 import synthetic
    ref = load_golden("full_2d_config")
    s = synthetic.survey_2d(seed=1234)
    tr = s.traces.cpu().numpy()
    assert hashlib.sha256(tr.astype(np.float32).tobytes()).hexdigest() == str(ref["input_sha256"])
    img, fold = _engine().migrate_bin_full(
        traces=tr, source_x=s.source_x, source_y=s.source_y, receiver_x=s.receiver_x,
        receiver_y=s.receiver_y, origin_x=s.origin_x, origin_y=s.origin_y,
        il_spacing=s.il_spacing, xl_spacing=s.xl_spacing, azimuth_deg=0.0, n_il=s.n_il,
        n_xl=s.n_xl, dt_ms=s.dt_ms, t_min_ms=s.t_min_ms, n_times=s.n_times,
        velocity_mps=s.velocity_mps, max_aperture_m=s.max_aperture_m,
        max_angle_deg=s.max_angle_deg, normalize=False)
    err = rel_l2(img, ref["image"])
    flips = np.abs(fold - ref["fold"]).sum()
    assert err <= FP32_TOL, err
    assert flips <= FOLD_FLIP_FRAC * ref["fold"].sum(), flips


def test_full_3d_20k_matches_reference():
    """20k traces x 500 samples -> 16 x 16 x 500 (golden made by running the
    reference's migrate_bin_full at constant V; input regenerated from its
    seed on the CPU and SHA-256 pinned)."""
    import hashlib
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import survey_3d_20k
    ref = load_golden("full_3d_20k")
    s = survey_3d_20k()
    tr = s.traces.numpy()
    assert hashlib.sha256(tr.astype(np.float32).tobytes()).hexdigest() == str(ref["input_sha256"])
    # 16-bit storage: the rounding of the stored samples (bf16 keeps 8
    # significant bits, f16 11 with a per-trace scale) sets the error
    for storage, tol in (("f32", FP32_TOL), ("bf16", 2e-3), ("f16", 3e-4)):
        from seisproc_b200.engine import MigrationEngine
        img, fold = MigrationEngine(storage=storage).migrate_bin_full(
            traces=tr, source_x=s.source_x, source_y=s.source_y, receiver_x=s.receiver_x,
            receiver_y=s.receiver_y, origin_x=s.origin_x, origin_y=s.origin_y,
            il_spacing=s.il_spacing, xl_spacing=s.xl_spacing, azimuth_deg=0.0, n_il=s.n_il,
            n_xl=s.n_xl, dt_ms=s.dt_ms, t_min_ms=0.0, n_times=s.n_times,
            velocity_mps=s.velocity_mps, max_aperture_m=s.max_aperture_m,
            max_angle_deg=s.max_angle_deg, normalize=False)
        err = rel_l2(img, ref["image"])
        flips = np.abs(fold - ref["fold"]).sum()
        assert err <= tol, (storage, err)
        assert flips <= max(2, FOLD_FLIP_FRAC * ref["fold"].sum()), (storage, flips)


def _small_3d(seed=3, n_traces=4000, lateral=True, utm=(0.0, 0.0), n_samples=200):
    from seisproc_b200 import synthetic
    return synthetic.survey_3d(n_traces=n_traces, seed=seed, n_samples=n_samples, extent=1600.0,
                               max_offset=1200.0, n_il=12, n_xl=10, spacing=25.0,
                               n_diffractors=12, aperture=500.0, lateral_velocity=lateral,
                               utm_origin=utm)


def _oracle_3d(s, **kw):
    n_t = s.n_times
    il = np.arange(s.n_il)[:, None]
    xl = np.arange(s.n_xl)[None, :]
    cx = (s.origin_x + il * s.il_spacing + 0 * xl).ravel()
    cy = (s.origin_y + 0 * il + xl * s.xl_spacing).ravel()
    t_ms = (np.arange(n_t, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    v = s.vrms.reshape(n_t, -1).astype(np.float64)
    return O.migrate_fp64(s.traces.cpu().numpy(), s.source_x, s.source_y, s.receiver_x,
                          s.receiver_y, cx, cy, t_ms, v, s.dt_ms, 0.0, s.max_aperture_m,
                          s.max_angle_deg, **kw)


def _engine_3d(s, storage="f32"):
    from seisproc_b200.engine import MigrationEngine
    eng = MigrationEngine(storage=storage)
    return eng.migrate_bin_full(
        traces=s.traces.cpu().numpy(), source_x=s.source_x, source_y=s.source_y,
        receiver_x=s.receiver_x, receiver_y=s.receiver_y, origin_x=s.origin_x,
        origin_y=s.origin_y, il_spacing=s.il_spacing, xl_spacing=s.xl_spacing, azimuth_deg=0.0,
        n_il=s.n_il, n_xl=s.n_xl, dt_ms=s.dt_ms, t_min_ms=0.0, n_times=s.n_times,
        max_aperture_m=s.max_aperture_m, max_angle_deg=s.max_angle_deg, normalize=False,
        velocity_model=s.vrms)


def test_vrms_3d_matches_fp64_oracle():
    s = _small_3d()
    img, fold = _engine_3d(s)
    oi, of = _oracle_3d(s)
    err = rel_l2(img.reshape(s.n_times, -1), oi)
    flips = np.abs(fold.reshape(s.n_times, -1) - of).sum()
    assert err <= FP32_TOL, err
    assert flips <= max(2, FOLD_FLIP_FRAC * of.sum()), flips


def test_utm_coordinates_float64_origin():
    """World coordinates near (5e5, 6e6) m: FP64 origin subtraction keeps FP32 accuracy."""
    s = _small_3d(utm=(5.0e5, 6.0e6))
    img, fold = _engine_3d(s)
    oi, of = _oracle_3d(s)
    assert rel_l2(img.reshape(s.n_times, -1), oi) <= FP32_TOL


@pytest.mark.parametrize("storage,tol", [("f16", 1e-3), ("bf16", 4e-3)])
def test_16bit_storage_error_vs_fp64(storage, tol):
    s = _small_3d(seed=4)
    img, _ = _engine_3d(s, storage=storage)
    oi, _ = _oracle_3d(s)
    err = rel_l2(img.reshape(s.n_times, -1), oi)
    assert err <= tol, f"{storage}: rel-L2 {err:.3e}"


def test_deterministic_bitwise():
    s = _small_3d(seed=5)
    a, fa = _engine_3d(s)
    b, fb = _engine_3d(s)
    assert np.array_equal(a, b) and np.array_equal(fa, fb)


def test_no_traces_gives_zero_image():
    from seisproc_b200.engine import MigrationEngine
    img, fold = MigrationEngine().migrate_bin_full(
        traces=np.zeros((100, 0), np.float32), source_x=np.zeros(0), source_y=np.zeros(0),
        receiver_x=np.zeros(0), receiver_y=np.zeros(0), origin_x=0, origin_y=0, il_spacing=25,
        xl_spacing=25, azimuth_deg=0, n_il=3, n_xl=2, dt_ms=4, t_min_ms=0, normalize=False)
    assert img.shape == (100, 3, 2) and not img.any() and not fold.any()


def test_traces_outside_aperture_contribute_nothing():
    from seisproc_b200.engine import MigrationEngine
    n = 50
    x = np.full(n, 1.0e5)
    img, fold = MigrationEngine().migrate_bin_full(
        traces=np.random.RandomState(0).randn(64, n).astype(np.float32), source_x=x,
        source_y=x, receiver_x=x, receiver_y=x, origin_x=0, origin_y=0, il_spacing=25,
        xl_spacing=25, azimuth_deg=0, n_il=4, n_xl=4, dt_ms=4, t_min_ms=0,
        max_aperture_m=1000, normalize=False)
    assert not img.any() and not fold.any()


def test_invalid_velocity_rejected():
    """A velocity that makes depth decrease with t0 is rejected by the device check."""
    s = _small_3d(seed=6, n_traces=500, n_samples=64)
    v = np.ascontiguousarray(s.vrms[::-1] * np.linspace(3, 1, s.n_times)[:, None, None],
                             dtype=np.float32)
    s.vrms = v
    with pytest.raises(ValueError):
        _engine_3d(s)


def test_normalize_by_fold_kat():
    """Known answers of the reference test (tests/test_kirchhoff_kernel.py:393-406)."""
    from seisproc_b200.kirchhoff import normalize_by_fold
    image = torch.tensor([[[10.0, 20.0], [30.0, 0.0]]])
    fold = torch.tensor([[[2.0, 4.0], [3.0, 0.0]]])
    n = normalize_by_fold(image, fold, min_fold=1)
    assert torch.allclose(n, torch.tensor([[[5.0, 5.0], [10.0, 0.0]]]))
    n2 = normalize_by_fold(torch.tensor([[[10.0, 20.0]]]), torch.tensor([[[1.0, 0.5]]]), 1)
    assert n2[0, 0, 0].item() == 10.0 and n2[0, 0, 1].item() == 20.0


def _plan_3d(s, in_t0_ms=0.0, **kw):
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan = PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                    origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                    xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                    in_t0_ms=in_t0_ms, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                    max_angle_deg=s.max_angle_deg, **kw)
    img, fold = plan.migrate(s.traces.cuda(), torch.from_numpy(s.vrms).cuda())
    plan.check()
    plan.close()
    return img.reshape(s.n_times, -1).cpu().numpy(), fold.reshape(s.n_times, -1).cpu().numpy()


@pytest.mark.parametrize("weight", ["obliquity_spreading", "spreading", "obliquity", "none"])
def test_weight_modes_match_fp64_oracle(weight):
    """Every weight mode (index-scaled and plain traveltime paths) vs FP64."""
    s = _small_3d(seed=6)
    img, fold = _plan_3d(s, weight=weight)
    oi, of = _oracle_3d(s, weight=weight)
    assert rel_l2(img, oi) <= FP32_TOL, weight
    assert np.abs(fold - of).sum() <= max(2, FOLD_FLIP_FRAC * of.sum())


def test_output_before_first_input_sample():
    """Input traces starting 40 ms after the output axis: indices below the first
    sample clamp to it (the low-clamp path), as the reference's clamp to
    [0, N - 1.001] does (kirchhoff_kernel.py:707-709)."""
    s = _small_3d(seed=7)
    img, fold = _plan_3d(s, in_t0_ms=40.0)
    n_t = s.n_times
    il = np.arange(s.n_il)[:, None]
    xl = np.arange(s.n_xl)[None, :]
    cx = (s.origin_x + il * s.il_spacing + 0 * xl).ravel()
    cy = (s.origin_y + 0 * il + xl * s.xl_spacing).ravel()
    t_ms = (np.arange(n_t, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    oi, of = O.migrate_fp64(s.traces.cpu().numpy(), s.source_x, s.source_y, s.receiver_x,
                            s.receiver_y, cx, cy, t_ms, s.vrms.reshape(n_t, -1), s.dt_ms, 40.0,
                            s.max_aperture_m, s.max_angle_deg)
    assert rel_l2(img, oi) <= FP32_TOL
    assert np.abs(fold - of).sum() <= max(2, FOLD_FLIP_FRAC * of.sum())


@pytest.mark.parametrize("weight", ["obliquity_spreading", "spreading", "obliquity", "none"])
def test_forward_only_rows_match_fp64_oracle(weight):
    """Plans built forward_only stage intercept-form float32 rows: the same
    operator to float rounding (vs the default plan and vs FP64)."""
    s = _small_3d(seed=6)
    img, fold = _plan_3d(s, weight=weight, forward_only=True)
    ref, rfold = _plan_3d(s, weight=weight)
    oi, of = _oracle_3d(s, weight=weight)
    assert rel_l2(img, oi) <= FP32_TOL, weight
    assert rel_l2(img, ref) <= 1e-5, weight
    assert np.array_equal(fold, rfold)


def test_forward_only_low_clamp_and_16bit():
    """The intercept frame under the low clamp (traces starting 40 ms late), and
    forward_only leaving 16-bit rows untouched."""
    s = _small_3d(seed=7)
    img, fold = _plan_3d(s, in_t0_ms=40.0, forward_only=True)
    ref, rfold = _plan_3d(s, in_t0_ms=40.0)
    assert rel_l2(img, ref) <= 1e-5 and np.array_equal(fold, rfold)
    b1, _ = _plan_3d(s, storage="bf16", forward_only=True)
    b0, _ = _plan_3d(s, storage="bf16")
    assert np.array_equal(b1, b0)


def test_forward_only_plan_refuses_gradient_and_mixed_batch():
    """A forward_only plan has no V-gradient, and a batch takes it only with
    other forward_only plans (the rows' form is one per launch)."""
    from seisproc_b200.batched import BatchedPSTM
    from seisproc_b200.kirchhoff import PSTMPlan
    s = _small_3d(seed=8, n_traces=1000)
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]

    def make(fo):
        return PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                        origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                        xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                        in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                        max_angle_deg=s.max_angle_deg, forward_only=fo)
    plan, other = make(True), make(False)
    v = torch.from_numpy(s.vrms).to(dev)
    img, _ = plan.migrate(s.traces.to(dev), v)
    with pytest.raises(Exception, match="forward_only"):
        plan.velocity_gradient(img, v)
    other.load_traces(s.traces.to(dev))
    with pytest.raises(Exception, match="forward_only"):
        BatchedPSTM([plan, other], v)
    b = BatchedPSTM([plan], v)
    b.migrate()
    b.check()
    assert torch.equal(b.images[0], img)
    b.close()
    other.close()
    d = plan.demigrate(img, v)  # still the adjoint, to ~1e-5
    assert d.shape == s.traces.shape
    plan.check()
    plan.close()


def test_plans_reuse_pooled_memory_and_trim():
    """Plans built and destroyed one after another take their memory from the
    library's pool; results stay the same, and trimming returns it."""
    import seisproc_b200
    from seisproc_b200 import synthetic
    from seisproc_b200.kirchhoff import PSTMPlan
    s = synthetic.survey_3d(n_traces=2000, seed=31, n_samples=150, extent=800.0,
                            max_offset=600.0, n_il=6, n_xl=6, spacing=25.0, n_diffractors=4,
                            aperture=300.0)
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    v = torch.from_numpy(s.vrms).to(dev)
    out = []
    for _ in range(3):
        p = PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                     origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                     xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                     in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                     max_angle_deg=s.max_angle_deg)
        img, fold = p.migrate(s.traces.to(dev), v)
        p.check()
        out.append((img.clone(), fold.clone()))
        p.close()
    for img, fold in out[1:]:
        assert torch.equal(img, out[0][0]) and torch.equal(fold, out[0][1])
    seisproc_b200.release_cached_memory()
    seisproc_b200.release_cached_memory(1 << 30)
    with pytest.raises(ValueError):
        seisproc_b200.release_cached_memory(-1)


@pytest.mark.parametrize("forward_only", [False, True])
def test_linearity_in_the_traces(forward_only):
    """The operator is linear in the trace samples: scaling the traces by a
    power of two scales the image exactly (no rounding enters: the staged rows,
    the interpolation and every partial sum scale with them), a sum of two
    trace sets migrates to the sum of their images within float32 rounding,
    and the fold does not depend on the samples.  Rows in intercept form
    (forward_only plans) interpolate as idx * slope + intercept, whose terms
    are up to a trace length larger than the sample, so their rounding is
    ~1e-5 of the image (within the 1e-4 parity tolerance); (x, dx) rows round
    at ~1e-7."""
    from seisproc_b200 import synthetic
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    s = synthetic.survey_3d(n_traces=40000, seed=11, n_samples=500, dt_ms=2.0, extent=2000.0,
                            max_offset=1500.0, n_il=64, n_xl=64, spacing=25.0, n_diffractors=20,
                            aperture=800.0)
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan = PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                    origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                    xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                    in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                    max_angle_deg=s.max_angle_deg, forward_only=forward_only)
    v = torch.from_numpy(s.vrms).to(dev)
    g = torch.Generator(device=dev).manual_seed(11)
    x = torch.randn((s.n_samples, s.n_traces), device=dev, generator=g)
    y = torch.randn((s.n_samples, s.n_traces), device=dev, generator=g)
    lx, fx = plan.migrate(x, v)
    lx = lx.clone()
    l4, f4 = plan.migrate(4.0 * x, v)
    assert torch.equal(l4, 4.0 * lx) and torch.equal(f4, fx)
    ly, _ = plan.migrate(y, v)
    ly = ly.clone()
    lxy, fxy = plan.migrate(x + y, v)
    plan.check()
    plan.close()
    assert torch.equal(fxy, fx)
    tol = 5e-5 if forward_only else 1e-6
    assert rel_l2(lxy.cpu().numpy(), (lx + ly).cpu().numpy()) <= tol


def test_reciprocity_and_translation():
    """Swapping every trace's source and receiver leaves the fold unchanged
    exactly and the image within float32 rounding (the traveltime, masks and
    weight are symmetric in the two legs, but the legs are summed in the other
    order: the float32 index moves by up to an ulp, 6e-5 of a sample at sample
    1000, which white-noise traces turn into ~1e-5 of the image, inside the
    1e-4 parity tolerance); moving the survey and the grid by a
    whole kilometre-scale offset leaves both bit for bit unchanged (the origin
    is subtracted in float64 before the float32 geometry is formed)."""
    from seisproc_b200 import synthetic
    from seisproc_b200.kirchhoff import PSTMPlan
    dev = torch.device("cuda")
    s = synthetic.survey_3d(n_traces=20000, seed=12, n_samples=400, dt_ms=2.0, extent=1600.0,
                            max_offset=1500.0, n_il=48, n_xl=40, spacing=25.0, n_diffractors=12,
                            aperture=700.0)
    v = torch.from_numpy(s.vrms).to(dev)
    tr = torch.from_numpy(np.random.RandomState(12).standard_normal(
        (s.n_samples, s.n_traces)).astype(np.float32)).to(dev)

    def run(sx, sy, rx, ry, ox, oy):
        c = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
             for a in (sx, sy, rx, ry)]
        p = PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=ox, origin_y=oy,
                     il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0, xl_dy=s.xl_spacing, t0_ms=0.0,
                     dt_ms=s.dt_ms, n_samples=s.n_samples, in_t0_ms=0.0, in_dt_ms=s.dt_ms,
                     max_aperture_m=s.max_aperture_m, max_angle_deg=s.max_angle_deg)
        img, fold = p.migrate(tr, v)
        p.check()
        p.close()
        return img.cpu().numpy(), fold.cpu().numpy()

    # coordinates on a 1/1024 m grid, so that the shifted ones are exact in float64
    g = [np.round(np.asarray(a, np.float64) * 1024.0) / 1024.0
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    img, fold = run(*g, s.origin_x, s.origin_y)
    assert fold.sum() > 0
    ri, rf = run(g[2], g[3], g[0], g[1], s.origin_x, s.origin_y)
    assert np.array_equal(rf, fold) and rel_l2(ri, img) <= 3e-5
    dx, dy = 512000.0, 6144000.0  # UTM-sized
    ti, tf = run(g[0] + dx, g[1] + dy, g[2] + dx, g[3] + dy, s.origin_x + dx, s.origin_y + dy)
    assert np.array_equal(tf, fold) and np.array_equal(ti, img)
