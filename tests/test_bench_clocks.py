"""The bench's clock record: NVML samples are summarised into the median SM
clock, the maximum and the throttle reasons seen (no device needed: the
samples are given)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_summary_of_nvml_samples():
    c = bench.ClockSampler(0)
    c.rows = [(1965.0, 1965.0, 0), (1950.0, 1965.0, 0x4), (1965.0, 1965.0, 0x1)]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]  # 0x1 (idle) is not a throttle reason


def test_summary_flags_slowdowns():
    c = bench.ClockSampler(0)
    c.rows = [(900.0, 1965.0, 0x8 | 0x40), (950.0, 1965.0, 0x20)]
    assert c.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_summary_without_samples():
    c = bench.ClockSampler(0)
    c.path = os.path.join(ROOT, "no-such-file.csv")
    assert c.summary()["reasons"] == ["unsampled"]
