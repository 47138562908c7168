"""bench.py's reference arm on the CPU at a small size: one JSON line with the
keys the benchmark contract names, rank 0 only, and the 'unavailable' line
for a workload the reference has no path for."""
import json
import os
import subprocess
import sys

from conftest import ROOT

SMALL = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--traces", "3000",
         "--samples", "100", "--grid", "20", "--crop", "2"]


def _run(extra, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *extra], cwd=ROOT,
                       capture_output=True, text=True, timeout=300, env=e)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_json_line():
    lines = _run(SMALL)
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e", "impl"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "Gpairs/s"
    assert d["higher_is_better"] is True and d["steps"] == 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "workload" in d["config"]


def test_reference_arm_other_ranks_print_nothing():
    assert _run(SMALL, env={"RANK": "1"}) == []


def test_reference_arm_unavailable_for_antialias():
    lines = _run(["--impl", "reference", "--antialias"])
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and "unavailable" in d


def test_time_rms_reference_arm_json_line():
    """--config time_rms --impl reference times the float32 oracle on the same
    workload with the same metric as the GPU arm."""
    lines = _run(["--config", "time_rms", "--impl", "reference", "--steps", "1", "--warmup",
                  "0", "--traces", "8000", "--samples", "100", "--grid", "20"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "time-domain RMS scatter Gevals/s"
    assert d["value"] > 0 and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("time-domain RMS operator, 8000 traces")


def test_velocity_reference_arm_and_unavailable_configs():
    lines = _run(["--config", "velocity", "--impl", "reference", "--steps", "1", "--warmup",
                  "0", "--samples", "100", "--grid", "20"])
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "V_rms grid Gsamples/s"
    assert d["value"] > 0 and "RegularGridInterpolator" in d["cpu_baseline"]["sample"]
    d = json.loads(_run(["--config", "lsq", "--impl", "reference"])[0])
    assert d["impl"] == "reference" and d["unavailable"]
    assert _run(["--config", "lsq", "--impl", "reference"], env={"RANK": "1"}) == []


def test_batched_reference_arm_json_line():
    """The batched config's reference arm: the reference algorithm migrating the
    classes one bin at a time on a crop, same metric as the GPU arm."""
    lines = _run(["--config", "batched", "--impl", "reference", "--steps", "1", "--warmup",
                  "0", "--classes", "3", "--samples", "100", "--grid", "20", "--crop", "2"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["metric"] == "PSTM Gpairs/s (out-sample x trace), batched classes"
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("batched 3D PSTM: 3 offset/azimuth classes")
    assert _run(["--config", "batched", "--impl", "reference", "--classes", "2"],
                env={"RANK": "1"}) == []
