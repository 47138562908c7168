"""The C-ABI library loads and exports every entry point include/*.h declares;
argument validation runs before any device work (no GPU needed)."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import ROOT


def _declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:pstm_status|int32_t|int64_t|void)\s+(pstm_\w+)\s*\(", src,
                            flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared_functions()
    assert "pstm_plan_create" in names and "pstm_migrate" in names
    assert len(names) >= 15


def test_library_exports_every_declared_symbol():
    from seisproc_b200 import _lib
    L = _lib.lib()
    missing = [n for n in _declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert L.pstm_abi_version() == 1


def test_plan_create_rejects_bad_config_without_device():
    from seisproc_b200 import _lib
    L = _lib.lib()
    grid = _lib.Grid(0, 1, 10, 0, 0, 25, 0, 0, 25, 0, 4)  # n_il = 0
    params = _lib.Params(100, 0, 4, 1000, 60, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    geo = _lib.Geometry(0, _lib.PSTM_F32, None, None, None, None)
    h = C.c_void_p()
    st = L.pstm_plan_create(C.byref(h), C.byref(grid), C.byref(params), C.byref(geo), None)
    assert st == _lib.PSTM_EINVAL
    assert "grid" in _lib.last_error()
    grid.n_il = 4
    params.max_angle_deg = 95.0
    assert L.pstm_plan_create(C.byref(h), C.byref(grid), C.byref(params), C.byref(geo),
                              None) == _lib.PSTM_EINVAL
    assert "max_angle_deg" in _lib.last_error()
    params.max_angle_deg = 60.0
    params.forward_only = 2
    assert L.pstm_plan_create(C.byref(h), C.byref(grid), C.byref(params), C.byref(geo),
                              None) == _lib.PSTM_EINVAL
    assert "forward_only" in _lib.last_error()
    params.forward_only = 0
    params.storage = 9
    assert L.pstm_plan_create(C.byref(h), C.byref(grid), C.byref(params), C.byref(geo),
                              None) == _lib.PSTM_EINVAL
    with pytest.raises(ValueError):
        _lib.check(_lib.PSTM_EINVAL)


def test_null_arguments_rejected():
    from seisproc_b200 import _lib
    L = _lib.lib()
    assert L.pstm_migrate_loaded(None, None, 0, 0, None, None, None) == _lib.PSTM_EINVAL
    assert L.pstm_normalize_by_fold(None, None, None, 0, 1.0, None) == _lib.PSTM_OK
    assert L.pstm_normalize_by_fold(None, None, None, 5, 1.0, None) == _lib.PSTM_EINVAL
    assert L.pstm_check(None, None) == _lib.PSTM_EINVAL
    # velocity grid: no model, then a 3-D model without its y tables
    assert L.pstm_velocity_grid(None, 2, 2, 1, None, None, 0, None, None, None, None, 0, None,
                                None) == _lib.PSTM_EINVAL
    one = C.c_void_p(16)  # never dereferenced: validation fails first
    assert L.pstm_velocity_grid(one, 2, 2, 3, one, one, 4, one, one, None, None, 4, one,
                                None) == _lib.PSTM_EINVAL
    assert "pstm_velocity_grid" in _lib.last_error()
