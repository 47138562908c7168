"""Cases run against the checked test build of the library (a separate
process started by tests/test_gpu_checked.py with SEISPSTM_LIBRARY=checked).

The checked build bounds-checks every staged-row shared address and every
trace-list entry inside the kernels, gives up bounded device waits after 50 ms,
and can simulate faults.  Each case prints one JSON line: clean runs agree with
the FP64 oracle and raise no flag; a simulated fault comes back as its status
(PSTM_EBOUNDS or PSTM_ETIMEOUT) with no GPU fault, and the next clean run in
the same process is correct again (the context stays usable).
"""
import json
import os
import sys

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import pstm_fp64 as O  # noqa: E402
from seisproc_b200 import _lib, synthetic  # noqa: E402
from seisproc_b200.kirchhoff import PSTMPlan  # noqa: E402


def survey():
    return synthetic.survey_3d(n_traces=6000, seed=12, n_samples=200, extent=1600.0,
                               max_offset=1200.0, n_il=12, n_xl=10, spacing=25.0,
                               n_diffractors=10, aperture=500.0)


def oracle(s, **kw):
    il = np.arange(s.n_il)[:, None]
    xl = np.arange(s.n_xl)[None, :]
    cx = (s.origin_x + il * s.il_spacing + 0 * xl).ravel()
    cy = (s.origin_y + 0 * il + xl * s.xl_spacing).ravel()
    t_ms = (np.arange(s.n_times, dtype=np.float32) * np.float32(s.dt_ms)).astype(np.float64)
    return O.migrate_fp64(s.traces.cpu().numpy(), s.source_x, s.source_y, s.receiver_x,
                          s.receiver_y, cx, cy, t_ms, s.vrms.reshape(s.n_times, -1), s.dt_ms, 0.0,
                          s.max_aperture_m, s.max_angle_deg, **kw)


def run(s, storage="f32", forward_only=True, antialias=False):
    """Migrates on the checked build; returns (status, image or None)."""
    dev = torch.device("cuda")
    c = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (s.source_x, s.source_y, s.receiver_x, s.receiver_y)]
    plan = PSTMPlan(*c, n_il=s.n_il, n_xl=s.n_xl, n_times=s.n_times, origin_x=s.origin_x,
                    origin_y=s.origin_y, il_dx=s.il_spacing, il_dy=0.0, xl_dx=0.0,
                    xl_dy=s.xl_spacing, t0_ms=0.0, dt_ms=s.dt_ms, n_samples=s.n_samples,
                    in_t0_ms=0.0, in_dt_ms=s.dt_ms, max_aperture_m=s.max_aperture_m,
                    max_angle_deg=s.max_angle_deg, storage=storage, forward_only=forward_only,
                    antialias=antialias, aa_dx=s.il_spacing, aa_dy=s.xl_spacing)
    try:
        plan.load_traces(s.traces.to(dev))
        img, _ = plan.migrate_loaded(torch.from_numpy(s.vrms).to(dev))
        torch.cuda.synchronize()
        try:
            plan.check()
        except _lib.PSTMError as e:
            return e.status, None
        return _lib.PSTM_OK, img.reshape(s.n_times, -1).cpu().numpy()
    finally:
        plan.close()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def main(case):
    assert _lib.CHECKED, "run with SEISPSTM_LIBRARY=checked"
    L = _lib.lib()
    s = survey()
    oi, _ = oracle(s)
    out = {"case": case}
    if case == "clean":
        for storage, fo in (("f32", True), ("f32", False), ("bf16", False), ("f16", False)):
            st, img = run(s, storage, fo)
            out[f"{storage}/{int(fo)}"] = [st, rel(img, oi) if img is not None else None]
        st, img = run(s, "f32", False, antialias=True)
        cols = list(range(0, s.n_il * s.n_xl, 7))  # the explicit-sum oracle is slow
        oa, _ = oracle(s, antialias=True, dx_out=s.il_spacing, dy_out=s.xl_spacing,
                       columns=cols)
        out["aa"] = [st, rel(img[:, cols], oa[:, cols]) if img is not None else None]
    else:
        kind = {"missing_copy": 1, "no_clamp": 2, "bad_list_entry": 3}[case]
        _lib.check(L.pstm_test_set_injection(kind))
        st, _ = run(s)
        _lib.check(L.pstm_test_set_injection(0))
        out["fault_status"] = st
        st2, img = run(s)  # the same process, after the fault
        out["after"] = [st2, rel(img, oi) if img is not None else None]
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main(sys.argv[1])
