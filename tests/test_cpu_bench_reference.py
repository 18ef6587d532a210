"""The bench's reference arm (`bench.py --impl reference`) on the CPU: one
JSON line with the contract's keys, timed on the oracle port; and the
`unavailable` line for the workload the reference has no path for."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *args],
                         cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_detect_line():
    d = _run("--workload", "detect_640x480", "--steps", "1", "--warmup", "3")
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["unit"] == "Mpix/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] in ("port", "reference") and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_unavailable_line():
    d = _run("--workload", "grad_16x1024x768")
    assert d["impl"] == "reference" and "unavailable" in d


def test_reference_schedule_stops_at_the_budget():
    """The reference arm's steps: all warm-up steps, then timed steps until the
    requested count or the wall-time budget (after at least one timed step)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert list(bench.RefSchedule(3, 4)) == [0, 1, 2, 3, 4, 5, 6]
    old = bench.REF_BUDGET_S
    try:
        bench.REF_BUDGET_S = -1.0  # already spent: one timed step, then stop
        assert list(bench.RefSchedule(3, 200)) == [0, 1, 2, 3]
    finally:
        bench.REF_BUDGET_S = old
