"""bench.py host logic without a GPU: the clock sampler's summary of the samples taken from the
start of the timed region on (median SM clock, maximum, throttle reasons)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _row(sm, mx=1965, hw="Not Active", hwt="Not Active", swt="Not Active", cap="Not Active"):
    return ["0", str(sm), str(mx), "900.0", "0x0", hw, hwt, swt, cap]


def test_clock_summary_keeps_the_timed_region():
    import bench
    c = bench.ClockSampler(0)
    assert c.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    # two warm-up samples (one throttled), then the timed region
    c.rows = [_row(1200, hwt="Active"), _row(1300), _row(1965), _row(1950, cap="Active"), _row(1965)]
    s = c.summary(2)
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]          # the thermal sample before the region is not counted
    assert c.summary(0)["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    assert c.summary(5)["reasons"] == ["unsampled"]  # no sample inside the region


def test_wait_rows_returns_without_a_sampler():
    import bench
    c = bench.ClockSampler(0)
    c.wait_rows(1, 5.0)          # no nvidia-smi process: returns at once
    assert c.rows == []
