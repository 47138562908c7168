"""The entry point that allocates no device memory, pstm_migrate_noalloc.

It serves callers that must not allocate while they run -- a process whose
caching allocator already owns the GPU's free memory, or a latency-critical
path that cannot take the device-wide synchronisation cudaFree implies.  Its
scratch is one static device array shared by every call.  This test calls it
through the C ABI twice in a row (different data each time, so the second call
runs on the first call's leftover scratch) and checks each result against the
plan-based entry point (pstm_plan_create + pstm_migrate) within the FP32
tolerance used by the other parity tests, and directly against the FP64
oracle.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import pstm_fp64 as O

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-4


def _case(seed):
    from seisproc_b200 import _lib, synthetic
    s = synthetic.survey_3d(n_traces=1200 + 100 * seed, seed=seed, n_samples=180, extent=900.0,
                            max_offset=600.0, n_il=9, n_xl=7, spacing=25.0, n_diffractors=5,
                            aperture=350.0)
    dev = torch.device("cuda")
    coords = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
              for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    grid = _lib.Grid(s.n_il, s.n_xl, s.n_times, s.origin_x, s.origin_y, s.il_spacing, 0.0, 0.0,
                     s.xl_spacing, 0.0, s.dt_ms)
    params = _lib.Params(s.n_samples, 0.0, s.dt_ms, s.max_aperture_m, s.max_angle_deg, 0,
                         _lib.WEIGHT_OBLIQUITY_SPREADING, _lib.CLAMP_FULL, _lib.PSTM_F32, 0, 0.0,
                         0.0, 0.0, 0)
    geo = _lib.Geometry(s.n_traces, _lib.PSTM_F64, *[c.data_ptr() for c in coords])
    vel = torch.from_numpy(s.vrms.reshape(s.n_times, -1)).to(dev)
    return s, coords, grid, params, geo, s.traces.to(dev).contiguous(), vel


def _plan_path(L, grid, params, geo, traces, vel, n_cols):
    from seisproc_b200 import _lib
    stream = torch.cuda.current_stream().cuda_stream
    h = C.c_void_p()
    _lib.check(L.pstm_plan_create(C.byref(h), C.byref(grid), C.byref(params), C.byref(geo),
                                  stream))
    img = torch.empty((grid.n_times, grid.n_il, grid.n_xl), device="cuda")
    fold = torch.empty_like(img)
    try:
        _lib.check(L.pstm_migrate(h, traces.data_ptr(), 0, vel.data_ptr(), n_cols, 1,
                                  img.data_ptr(), fold.data_ptr(), stream))
        _lib.check(L.pstm_check(h, stream))
    finally:
        L.pstm_plan_destroy(h)
    return img, fold


def _noalloc(L, grid, params, geo, traces, vel, n_cols):
    from seisproc_b200 import _lib
    img = torch.full((grid.n_times, grid.n_il, grid.n_xl), float("nan"), device="cuda")
    fold = torch.full_like(img, -1.0)
    torch.cuda.synchronize()
    _lib.check(L.pstm_migrate_noalloc(C.byref(grid), C.byref(params), C.byref(geo),
                                      traces.data_ptr(), vel.data_ptr(), n_cols, 1,
                                      img.data_ptr(), fold.data_ptr(),
                                      torch.cuda.current_stream().cuda_stream))
    return img, fold


def test_noalloc_matches_plan_entry_point_on_two_calls():
    from seisproc_b200 import _lib
    L = _lib.lib()
    for seed in (21, 22):
        s, coords, grid, params, geo, traces, vel = _case(seed)
        n_cols = s.n_il * s.n_xl
        ref_img, ref_fold = _plan_path(L, grid, params, geo, traces, vel, n_cols)
        img, fold = _noalloc(L, grid, params, geo, traces, vel, n_cols)
        assert torch.isfinite(img).all()
        err = rel_l2(img.cpu().numpy(), ref_img.cpu().numpy())
        assert err <= FP32_TOL, (seed, err)
        assert torch.equal(fold, ref_fold), seed
        oi, of = _fp64(s)
        assert rel_l2(img.reshape(s.n_times, -1).cpu().numpy(), oi) <= FP32_TOL, seed
        assert np.abs(fold.reshape(s.n_times, -1).cpu().numpy() - of).sum() <= 2, seed


def _fp64(s):
    il = np.arange(s.n_il)[:, None]
    xl = np.arange(s.n_xl)[None, :]
    cx = (s.origin_x + il * s.il_spacing + 0 * xl).ravel()
    cy = (s.origin_y + 0 * il + xl * s.xl_spacing).ravel()
    t_ms = (np.arange(s.n_times, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    return O.migrate_fp64(s.traces.cpu().numpy(), s.source_x, s.source_y, s.receiver_x,
                          s.receiver_y, cx, cy, t_ms, s.vrms.reshape(s.n_times, -1), s.dt_ms,
                          0.0, s.max_aperture_m, s.max_angle_deg)


def test_noalloc_rejects_problems_beyond_its_scratch():
    """Short traces, so the staged kernel fits, but enough traces that the
    worst-case tile lists and staged rows exceed the scratch array: the call is
    rejected before any launch (the coordinates are never read)."""
    from seisproc_b200 import _lib
    L = _lib.lib()
    s, coords, grid, params, geo, traces, vel = _case(23)
    n_big = 40_000
    zeros = torch.zeros(n_big, dtype=torch.float64, device="cuda")
    big_geo = _lib.Geometry(n_big, _lib.PSTM_F64, *([zeros.data_ptr()] * 4))
    big_tr = torch.zeros((s.n_samples, n_big), device="cuda")
    st = L.pstm_migrate_noalloc(C.byref(grid), C.byref(params), C.byref(big_geo),
                                big_tr.data_ptr(), vel.data_ptr(), s.n_il * s.n_xl, 1,
                                traces.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert st == _lib.PSTM_EINVAL
    assert "scratch" in _lib.last_error()


def test_noalloc_rejects_non_finite_coordinates():
    from seisproc_b200 import _lib
    L = _lib.lib()
    s, coords, grid, params, geo, traces, vel = _case(24)
    coords[0][5] = float("nan")
    img = torch.empty((grid.n_times, grid.n_il, grid.n_xl), device="cuda")
    st = L.pstm_migrate_noalloc(C.byref(grid), C.byref(params), C.byref(geo), traces.data_ptr(),
                                vel.data_ptr(), s.n_il * s.n_xl, 1, img.data_ptr(), None,
                                torch.cuda.current_stream().cuda_stream)
    assert st == _lib.PSTM_EINVAL
    assert "non-finite" in _lib.last_error()
