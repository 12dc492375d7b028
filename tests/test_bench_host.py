"""Host-side pieces of bench.py that its JSON line depends on: the clock and
throttle-reason summary, the stdout guard around the reference's progress
prints, and the algorithmic-byte count of the RK3 roofline."""
import ctypes
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_clock_summary_reports_median_max_and_active_reasons():
    cs = bench.ClockSampler(0)
    # index, clocks.sm, clocks.max.sm, power, active mask, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    cs.rows = [["0", "1965", "1965", "400.5", "0x0", "Not Active", "Not Active", "Not Active", "Not Active"],
               ["0", "1800", "1965", "990.0", "0x4", "Not Active", "Not Active", "Not Active", "Active"],
               ["0", "1900", "1965", "700.0", "0x0", "Not Active", "Not Active", "Not Active", "Not Active"]]
    s = cs.summary()
    assert s["sm_mhz"] == 1900.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert s["power_w_max"] == 990.0 and s["samples"] == 3
    assert bench.ClockSampler(0).summary()["reasons"] == ["unsampled"]


def test_reference_progress_prints_stay_off_stdout(capfd):
    libc = ctypes.CDLL(None)
    with bench.c_stdout_to_stderr():
        libc.printf(b"\r[progress] t = 0.5")
    out, err = capfd.readouterr()
    assert "[progress]" not in out
    assert "[progress]" in err
    print('{"metric": "x"}')
    out, _ = capfd.readouterr()
    assert out == '{"metric": "x"}\n'


def test_rk3_algorithmic_bytes():
    # 600 state values x b_s + 3 stages x (10 geometry values x b_g + 32 bytes of neighbour rows)
    assert bench.algorithmic_bytes_per_step(1, 4, 4) == 600 * 4 + 3 * (40 + 32)
    assert bench.algorithmic_bytes_per_step(1, 8, 8) == 600 * 8 + 3 * (80 + 32)
    assert bench.algorithmic_bytes_per_step(5308416, 4, 4) == 5308416 * 2616
