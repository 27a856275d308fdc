"""bench.py's host-side contract on CPU: the reference arm (--impl reference: the oracle port
timed on the host cores) prints one JSON line with the contract's keys."""
import argparse
import io
import json
import os
import sys
from contextlib import redirect_stdout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_prints_one_contract_line(monkeypatch):
    """Two steps of the oracle loop at 2^14 rays (the arm's own schedule, shortened here): the
    line carries impl, value, unit, cpu_baseline (kind port, cores) and a zero-copy e2e."""
    monkeypatch.setattr(bench, "REF_STEPS", 2)
    monkeypatch.setattr(bench, "RAYS", 1 << 14)
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    args = argparse.Namespace(gpus=1, steps=20, warmup=5, impl="reference")
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    lines = [ln for ln in buf.getvalue().splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["value"] > 0
    assert d["steps"] >= 1 and d["warmup"] == 1 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["metric"] == bench.METRIC and d["config"]["workload"]
