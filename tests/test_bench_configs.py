"""The default bench line's `configs` object: each other workload runs as its
own `bench.py --workload W` process and the summary keeps its value, step
time, end-to-end rate, clocks and parity. Checked on the CPU with the
subprocess replaced by canned results (a line, a failing run, a timeout)."""

from __future__ import annotations

import json
import os
import subprocess
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_other_configs_summary(monkeypatch):
    calls = []

    def fake_run(cmd, **kw):
        name = cmd[cmd.index("--workload") + 1]
        calls.append(cmd)
        assert "--no-cpu-baseline" in cmd and kw["timeout"] == bench.OTHER_TIMEOUT_S
        if name == "mc_cascade":
            return subprocess.CompletedProcess(cmd, 1, "", "progress\nRuntimeError: no device\n")
        if name == "beam_scheme":
            raise subprocess.TimeoutExpired(cmd, kw["timeout"])
        line = {"metric": "m", "value": 2.0, "unit": "u", "ms_per_step": 3.0, "steps": 5, "warmup": 3,
                "dtype": "f32", "config": {"workload": name + "_w"}, "e2e": {"value": 1.5},
                "parity": {"checked": True, "candidates_match": True}, "clocks": {"sm_mhz": 1965.0}}
        return subprocess.CompletedProcess(cmd, 0, "noise\n" + json.dumps(line) + "\n", "")

    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    out = bench.other_configs()
    assert [c[c.index("--workload") + 1] for c in calls] == [n for n, _, _ in bench.OTHER_CONFIGS]
    for name, steps, warmup in bench.OTHER_CONFIGS:
        assert warmup >= 3
        rec = out[name]
        if name == "mc_cascade":
            assert rec["rc"] == 1 and rec["error"] == "RuntimeError: no device"
        elif name == "beam_scheme":
            assert rec["rc"] is None and "timed out" in rec["error"]
        else:
            assert rec["rc"] == 0 and rec["workload"] == name + "_w"
            assert rec["value"] == 2.0 and rec["e2e"] == 1.5 and rec["parity"]["candidates_match"]
