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
    # the scope table's figure per element and step: 660 b_s + 30 b_g + 60
    # (FP64 5,580 B, FP32 2,820 B)
    assert bench.algorithmic_bytes_per_step(1, 4, 4) == 2820
    assert bench.algorithmic_bytes_per_step(1, 8, 8) == 5580
    assert bench.algorithmic_bytes_per_step(5308416, 4, 4) == 5308416 * 2820
    # the kernel's own minimum: k2 not written in the last stage, 32-byte records
    assert bench.tight_bytes_per_step(1, 4, 4) == 600 * 4 + 3 * (40 + 32) == 2616
    assert bench.tight_bytes_per_step(1, 8, 8) == 600 * 8 + 3 * (80 + 32) == 5136


def test_kinetic_algorithmic_bytes():
    # 2 x 240 b_s + 10 b_g + 20 per element and step
    assert bench.kinetic_algorithmic_bytes(1, 4, 4) == 2 * 240 * 4 + 40 + 20
    assert bench.kinetic_algorithmic_bytes(1, 8, 8) == 2 * 240 * 8 + 80 + 20
