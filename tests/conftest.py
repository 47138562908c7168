import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

# the kernel-shape tuner's cache: one file per test session, inherited by the
# subprocesses the tests start, never the user's
import tempfile  # noqa: E402

os.environ.setdefault("SEISPSTM_TUNE_CACHE",
                      os.path.join(tempfile.gettempdir(), f"seispstm_tune_tests_{os.getpid()}.json"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (B200) device and libseispstm.so")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def golden_grid(d):
    """Unpack the grid vector stored by make_golden.py."""
    g = d["grid"]
    ox, oy, dx, dy, nil, nxl, dt, tmin, v, A, ang = [float(x) for x in g[:11]]
    return dict(origin_x=ox, origin_y=oy, il_spacing=dx, xl_spacing=dy, n_il=int(nil),
                n_xl=int(nxl), dt_ms=dt, t_min_ms=tmin, velocity_mps=v, max_aperture_m=A,
                max_angle_deg=ang)


@pytest.fixture
def golden():
    return load_golden
