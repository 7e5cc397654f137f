"""bench.py's reference arm runs on the host (the reference's own step,
compiled from its sources): its JSON line keeps the contract's keys."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _run(*args):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line_plain(have_ref):
    d = _run("--impl", "reference", "--workload", "plain", "--steps", "1", "--warmup", "3")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "cell-updates/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("plain")


def test_reference_arm_sweep_is_unavailable():
    d = _run("--impl", "reference", "--workload", "sweep64", "--steps", "1")
    assert d["impl"] == "reference" and "unavailable" in d


def test_reference_arm_warm_start_is_unavailable():
    # the reference has no warm start: its cold solves appear as the
    # workload's projected CPU baseline instead
    d = _run("--impl", "reference", "--workload", "warm_start", "--steps", "1")
    assert d["impl"] == "reference" and "unavailable" in d
