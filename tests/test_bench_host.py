"""Host logic of bench.py that needs no GPU: the summary of the nvidia-smi clock
samples taken during the timed region (median SM clock, max clock, throttle
reasons seen active)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _line(sm, smax, active="0x0000000000000000", hw="Not Active", hwt="Not Active", swt="Not Active",
          cap="Not Active", power="650.1"):
    return ", ".join([str(sm), str(smax), power, active, hw, hwt, swt, cap])


def test_clean_run():
    lines = [_line(1965, 1965), _line(1950, 1965), _line(1965, 1965)]
    out = bench.ClockSampler.summarize(lines)
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}


def test_reasons_are_collected_and_sorted():
    lines = [_line(1300, 1965, cap="Active"), _line(1290, 1965, hwt="Active", cap="Active"),
             _line(1310, 1965)]
    out = bench.ClockSampler.summarize(lines)
    assert out["sm_mhz"] == 1300.0
    assert out["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_malformed_lines_are_skipped_whole():
    lines = ["", "garbage", _line("[N/A]", 1965), _line(1800, "[N/A]", cap="Active"), _line(1900, 1965)]
    out = bench.ClockSampler.summarize(lines)
    assert out == {"sm_mhz": 1900.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 1}


def test_no_samples():
    out = bench.ClockSampler.summarize([])
    assert out["sm_mhz"] is None and out["samples"] == 0 and out["reasons"] == []
