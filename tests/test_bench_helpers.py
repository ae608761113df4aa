"""bench.py's timing helpers on CPU: the clock sampler keeps the rows read inside the timed region (else the last one
before it), reports the median SM clock and the throttle reasons that were active, and says when nothing was
sampled; the percentile helper picks the nearest-rank value."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def row(sm, reasons=()):
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    return ["0", str(sm), "1965", "700.0", "0x0"] + ["Active" if n in reasons else "Not Active" for n in names]


def test_clock_sampler_summary():
    c = bench.ClockSampler(0)
    c.t0, c.t1 = 10.0, 10.5
    c.rows = [(9.9, row(1200)), (10.1, row(1965)), (10.3, row(1950, ("sw_power_cap",))), (10.45, row(1965))]
    s = c.summary()
    assert s["samples_in_region"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    c.rows = [(9.8, row(1500)), (9.9, row(1800, ("hw_slowdown",)))]  # nothing inside: the last row before it
    s = c.summary()
    assert s["samples_in_region"] == 0 and s["samples"] == 1 and s["sm_mhz"] == 1800.0 and s["reasons"] == ["hw_slowdown"]
    c.rows = []
    assert c.summary()["reasons"] == ["unsampled"]


def test_percentile_nearest_rank():
    v = sorted(float(x) for x in range(1, 101))
    assert bench.percentile(v, 0.5) == 50.0 and bench.percentile(v, 0.99) == 99.0 and bench.percentile(v, 1.0) == 100.0
    assert bench.percentile([3.0], 0.999) == 3.0


def test_tail_order_keeps_every_key_and_ends_with_the_headline_figures():
    line = {"metric": "m", "value": 1.0, "serve": {"x": 1}, "p99_ms": 0.2, "batching": {}, "clocks": {}, "unit": "u"}
    out = bench.tail_order(line)
    assert out == line
    keys = list(out)
    assert keys[:4] == ["metric", "serve", "batching", "unit"] and keys[-1] == "value"
