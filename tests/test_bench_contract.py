"""bench.py's JSON contract on the CPU: the reference arm names the case it actually ran (the
bounded CPU sample of the device workload), and the clock summary covers only the samples taken
while the timed region ran."""
import argparse
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_names_the_sample_it_ran(monkeypatch, capsys):
    cells = bench.CPU_SAMPLE_SIDE ** 3
    fake = {"value": 1.0e4, "unit": "cell-iters/s", "cores": 1, "kind": "reference", "sample": "test",
            "cells": cells}
    seen = {}

    def fake_baseline(**kw):
        seen.update(kw)
        return fake

    monkeypatch.setattr(bench, "cpu_baseline", fake_baseline)
    monkeypatch.delenv("RANK", raising=False)
    args = argparse.Namespace(gpus=1, steps=10, warmup=3, cells=1_000_000)
    bench.run_reference(args)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    # the config describes the sample that ran, not the device arm's 1M-cell case
    assert line["config"]["cells"] == cells == line["cpu_baseline"]["cells"]
    assert str(cells) in line["config"]["workload"]
    assert "1000000" in line["config"]["sample_of"]
    assert line["metric"] == bench.METRIC and line["unit"] == "cell-iters/s" and line["higher_is_better"] is True
    assert line["e2e"] == {"value": 1.0e4, "unit": "cell-iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert seen["iterations"] == 6  # min(K, 5) timed outer iterations plus the excluded first one
    assert line["steps"] == 5 and abs(line["ms_per_step"] - cells / 1.0e4 * 1e3) < 1e-9


def test_reference_arm_other_ranks_print_nothing(monkeypatch, capsys):
    monkeypatch.setattr(bench, "cpu_baseline", lambda **kw: (_ for _ in ()).throw(AssertionError("ran")))
    monkeypatch.setenv("RANK", "1")
    bench.run_reference(argparse.Namespace(gpus=2, steps=10, warmup=3, cells=1_000_000))
    assert capsys.readouterr().out == ""


def test_clock_summary_uses_samples_from_the_timed_region():
    c = bench.ClockSampler(0)
    idle = ["0", "345", "1965", "120", "0x0", "Not Active", "Not Active", "Not Active", "Not Active"]
    busy = ["0", "1965", "1965", "950", "0x4", "Not Active", "Not Active", "Not Active", "Active"]
    c.rows = [idle, busy, busy]
    c.start = 1
    s = c.summary()
    assert s == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 2}
    c.rows, c.start = [], 0
    assert c.summary()["reasons"] == ["unsampled"]
