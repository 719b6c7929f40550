"""bench.py's reference arm on the CPU: every step a bounded band of the 12 MP
frame sized from the run's step count, timed and scaled to ms per frame, and
the JSON line the driver reads (impl, metric, unit, cpu_baseline, e2e with no
host copies).  The band budget is shrunk so that the test runs in seconds."""
import argparse
import contextlib
import io
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(bench, "REFERENCE_ARM_BUDGET_S", 0.2)
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        assert bench.reference_arm(argparse.Namespace(gpus=1, steps=2, warmup=1)) == 0
    line = json.loads(out.getvalue().strip().splitlines()[-1])
    assert line["impl"] == "reference"
    if "unavailable" in line:  # the reference build is absent: the arm says so and exits 0
        return
    assert line["metric"] == bench.METRIC and line["unit"] == "ms/frame" and line["steps"] == 2
    assert line["value"] > 0 and line["higher_is_better"] is False
    sample = line["cpu_baseline"]["sample"]
    assert "band of the frame" in sample and "4032x16 " in sample  # the smallest band at this budget
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "ms/frame", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "full_chain_12mp_4032x3024"


def test_reference_arm_other_ranks_do_no_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        assert bench.reference_arm(argparse.Namespace(gpus=2, steps=2, warmup=1)) == 0
    assert out.getvalue() == ""
