"""Host-side parts of bench.py on the CPU: the reference arm's JSON line (the
fields a driver reads), the time-to-solution formula and the repetition of
the CPU baseline's sample."""
import json
import math
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_t99_is_the_reference_formula():
    # openjij/utils/benchmark.py:205-224: tau * ln(1 - 0.99) / ln(1 - p_s)
    assert bench._t99(10.0, 0.5) == pytest.approx(10.0 * math.log(0.01) / math.log(0.5))
    # deviation (stated in bench._t99): the reference gives 0 at p_s = 1
    # (benchmark.py:216-217), here the time of the one call, tau
    assert bench._t99(3.0, 1.0) == 3.0
    assert bench._t99(3.0, 0.0) == float("inf")


def test_repeat_for_accumulates_until_the_budget():
    calls = []

    def sample():
        calls.append(1)
        return 1000.0, 0.25  # 1000 attempts/s for 0.25 s

    v, seconds, reps = bench._repeat_for(sample, min_seconds=1.0)
    assert reps == 4 and len(calls) == 4
    assert seconds == pytest.approx(1.0) and v == pytest.approx(1000.0)
    # one sample at least, even with no budget
    v, seconds, reps = bench._repeat_for(sample, min_seconds=0.0)
    assert reps == 1 and seconds == pytest.approx(0.25)


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "1",
                          "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "spin-flip attempts/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    assert line["e2e"] == {"value": line["value"], "unit": "attempts/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["config"]["workload"] == "dense_ising_N100_R100_S1000"
    # the same workload keys as the GPU arm's line
    assert line["config"] == json.loads(json.dumps(bench._config_of(bench._workload(1))))


_MAPS_PROBE = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--config", "1", "--steps", "1", "--warmup", "0"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit:
    pass
maps = open("/proc/self/maps").read()
print("MAPS", int("libojb200" in maps), int("_cxxjij" in maps), int("liboj_oracle" in maps))
"""


def test_reference_arm_maps_no_product_library():
    """The reference arm runs the oracle's restatement of the reference's CPU
    path only: after a whole run the process has mapped the oracle's library
    and neither of the product's shared objects."""
    out = subprocess.run([sys.executable, "-c", _MAPS_PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    tag = [ln for ln in out.stdout.splitlines() if ln.startswith("MAPS")][-1].split()
    assert tag[1:] == ["0", "0", "1"], tag


def test_other_configs_summary_reads_each_line_and_reports_failures(monkeypatch):
    """The default line's configs 1 and 3-6 come from one bench.py process per
    config: the last JSON line of each is summarised, and a config whose
    process fails is reported as an error (not left out)."""
    line = {"config": {"workload": "w"}, "kernel": {"name": "k"}, "value": 2.0, "unit": "attempts/s",
            "ms_per_step": 1.5, "e2e": {"value": 1.0}, "clocks": {"sm_mhz": 1965.0},
            "roofline": {"kernel_ms": 1.2, "bound": "issue", "frac": 0.5, "field_drift": None}}
    seen = []

    def fake_run(cmd, capture_output, text, timeout, check):
        c = int(cmd[cmd.index("--config") + 1])
        seen.append(c)
        assert "--no-cpu" in cmd and "--no-tts" in cmd
        if c == 4:
            raise subprocess.CalledProcessError(1, cmd)
        return subprocess.CompletedProcess(cmd, 0, stdout="noise\n" + json.dumps(line) + "\n", stderr="")

    monkeypatch.setattr(subprocess, "run", fake_run)
    out = bench.other_configs_summary(steps=2, warmup=3)
    assert seen == [1, 3, 4, 5, 6]
    assert set(out) == {"config1", "config3", "config4", "config5", "config6"}
    assert "error" in out["config4"]
    assert out["config3"]["value"] == 2.0 and out["config3"]["kernel"] == "k"
    assert out["config3"]["roofline_bound"] == "issue" and out["config3"]["roofline_frac"] == 0.5
