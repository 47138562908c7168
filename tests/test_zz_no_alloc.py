"""The entry point that allocates no device memory, pstm_migrate_noalloc.

It serves callers that must not allocate while they run -- a process whose
caching allocator already owns the GPU's free memory, or a latency-critical
path that cannot take the device-wide synchronisation cudaFree implies.  Its
scratch is one static device array shared by every call.  This test calls it
through the C ABI twice in a row (different data each time, so the second call
runs on the first call's leftover scratch) and checks each result against the
plan-based entry point (pstm_plan_create + pstm_migrate) within the FP32
tolerance used by the other parity tests.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_l2

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


def test_noalloc_rejects_problems_beyond_its_scratch():
    from seisproc_b200 import _lib
    L = _lib.lib()
    s, coords, grid, params, geo, traces, vel = _case(23)
    big = _lib.Params(200_000, 0.0, s.dt_ms, s.max_aperture_m, s.max_angle_deg, 0, 0, 0, 0, 0,
                      0.0, 0.0, 0.0, 0)
    st = L.pstm_migrate_noalloc(C.byref(grid), C.byref(big), C.byref(geo), traces.data_ptr(),
                                vel.data_ptr(), s.n_il * s.n_xl, 1, traces.data_ptr(), None,
                                torch.cuda.current_stream().cuda_stream)
    assert st == _lib.PSTM_EINVAL
    assert "scratch" in _lib.last_error() or "too long" in _lib.last_error()
