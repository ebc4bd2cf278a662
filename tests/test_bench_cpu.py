"""bench.py helpers that need no GPU: the clock sampler's summary keeps only
the samples taken inside the timed region, and the whole-job rate divides by
every replica's solves."""
import bench


def _row(sm, reasons=()):
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    return ["0", str(sm), "1965", "700.0", "0x0"] + ["Active" if n in reasons else "Not Active" for n in names]


def test_clock_summary_uses_the_samples_of_the_timed_region():
    c = bench.ClockSampler(0)
    # a sample before the region (a throttled start-up) and three inside it
    c.rows = [_row(1200, ("sw_thermal_slowdown",)), _row(1965), _row(1950, ("sw_power_cap",)), _row(1965)]
    c.first = 1
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_summary_without_samples_in_the_region():
    c = bench.ClockSampler(0)
    c.rows, c.first = [_row(1965)], 1  # nothing arrived inside: the last sample before it stands in
    assert c.summary()["samples"] == 1
    c.rows, c.first = [], 0
    assert c.summary()["reasons"] == ["unsampled"]


def test_job_rate_counts_every_replica():
    assert bench.job_ms_per_solve(800.0, 1, 10) == 80.0
    assert bench.job_ms_per_solve(800.0, 4, 10) == 20.0
