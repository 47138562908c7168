"""The checked test build of the library (libseispstm_checked.so, built by
``build(checked=True)``): kernels that bounds-check every staged-row shared
address and every trace-list entry, bounded device waits of 50 ms, and
simulated faults.  Each case runs tests/checked_cases.py in its own process
(SEISPSTM_LIBRARY=checked).  Clean runs must match the FP64 oracle with no
flag raised; a stage copy that is never issued must come back as
PSTM_ETIMEOUT, an index past the staged row or a corrupt list entry as
PSTM_EBOUNDS -- caught by the checks, with no GPU fault -- and the next run in
the same process must be correct."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _case(name):
    env = dict(os.environ, SEISPSTM_LIBRARY="checked")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_cases.py"), name],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])


def test_checked_build_clean_runs_match_oracle():
    from seisproc_b200 import _lib
    d = _case("clean")
    tol = {"f32/1": 1e-4, "f32/0": 1e-4, "bf16/0": 4e-3, "f16/0": 1e-3, "aa": 1e-4}
    for k, t in tol.items():
        status, err = d[k]
        assert status == _lib.PSTM_OK, (k, status)
        assert err <= t, (k, err)


@pytest.mark.parametrize("case,status", [("missing_copy", 3), ("no_clamp", 4),
                                         ("bad_list_entry", 4)])
def test_simulated_fault_reports_status_and_recovers(case, status):
    from seisproc_b200 import _lib
    assert (_lib.PSTM_ETIMEOUT, _lib.PSTM_EBOUNDS) == (3, 4)
    d = _case(case)
    assert d["fault_status"] == status, d
    st, err = d["after"]
    assert st == _lib.PSTM_OK and err <= 1e-4, d
