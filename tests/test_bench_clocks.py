"""bench.py's clock record (ClockSampler.summary) from nvidia-smi samples, on fake CSV lines: the
median SM clock, the maximum, and the throttle reasons seen active at any sample."""

import os
import shutil

import bench


def _summary(tmp_path, lines):
    s = bench.ClockSampler(0)
    s.path = os.path.join(tmp_path, "clocks.csv")
    with open(s.path, "w") as f:
        f.write("\n".join(lines) + "\n")
    s.proc = object()  # as if nvidia-smi had run
    return s.summary()


def test_median_max_and_reasons(tmp_path):
    lines = ["1965, 1965, 610.2, Not Active, Not Active, Not Active, Not Active",
             "1950, 1965, 980.0, Not Active, Not Active, Not Active, Active",
             "1965, 1965, 990.5, Not Active, Not Active, Not Active, Active",
             "[N/A], 1965, 12.0, Not Active, Not Active, Not Active, Not Active",  # unreadable sample
             "garbage"]
    d = _summary(tmp_path, lines)
    assert d["samples"] == 3 and d["sm_mhz"] == 1965.0 and d["sm_max_mhz"] == 1965.0
    assert d["reasons"] == ["sw_power_cap"]


def test_slowdown_reasons_are_reported(tmp_path):
    d = _summary(tmp_path, ["1200, 1965, 700, Active, Not Active, Active, Not Active"])
    assert d["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"] and d["sm_mhz"] == 1200.0


def test_no_samples_no_record(tmp_path):
    assert _summary(tmp_path, []) is None
    if shutil.which("nvidia-smi") is None:
        with bench.ClockSampler(0) as s:
            pass
        assert s.summary() is None
