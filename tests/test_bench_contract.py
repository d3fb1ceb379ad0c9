"""CPU checks of bench.py's reference arm: one JSON line with the contract's keys
on rank 0, nothing (exit 0) on the other ranks of a multi-process launch."""
import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _run(extra_env, *args):
    env = dict(os.environ, OPENBLAS_NUM_THREADS=os.environ.get("OPENBLAS_NUM_THREADS", "4"), **extra_env)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", *args], cwd=ROOT,
                          env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    out = _run({}, "--workload", "sm_water32", "--steps", "1", "--warmup", "0")
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is False and d["steps"] == 1
    assert d["value"] > 0 and abs(d["ms_per_step"] - 1e3 * d["value"]) < 1e-6 * d["ms_per_step"]
    assert "workload" in d["config"] and d["data"] == "synthetic"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    out = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--workload", "sm_water32", "--steps", "1",
               "--warmup", "0")
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_reports_the_calls_it_timed():
    """With a budget smaller than one call, exactly one whole call is timed and
    the line says so (steps 1, the request kept beside it); no scaled sample."""
    out = _run({}, "--workload", "sm_water32", "--steps", "5", "--warmup", "0", "--ref-budget", "0.001")
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][0])
    assert d["steps"] == 1 and d["requested_steps"] == 5
    assert len(d["timed_calls_s"]) == 1 and d["value"] == d["timed_calls_s"][0]
    assert "whole" in d["cpu_baseline"]["sample"] and "scaled" not in d["cpu_baseline"]["sample"]


def test_timed_calls_stops_at_the_budget_or_the_steps():
    sys.path.insert(0, str(ROOT))
    import bench
    calls = []
    times, w = bench.timed_calls(lambda: calls.append(1), 4, lambda: None, 2, 1e9)
    assert len(times) == 4 and w == 2 and len(calls) == 4
    import time as _t
    times, _ = bench.timed_calls(lambda: _t.sleep(0.05), 10, lambda: None, 0, 0.12)
    assert 1 <= len(times) < 10


def test_reference_arm_unavailable_where_the_oracle_does_not_fit():
    """The 2048-H2O submatrix workload has no CPU restatement run (full 47104 x 47104
    matrices): the arm prints one 'unavailable' line and exits 0 without building it."""
    out = _run({}, "--workload", "sm_water2048", "--steps", "1", "--warmup", "0")
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and "host memory" in d["unavailable"]
