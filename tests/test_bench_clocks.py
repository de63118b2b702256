"""The benchmark's clock record: nvidia-smi samples stamped by nvidia-smi are
matched to the timed window on the host clock; a window shorter than the
sampling period takes the nearest sample on each side; throttle reasons are
collected from every sample used."""
import importlib.util
import os
import time

_spec = importlib.util.spec_from_file_location(
    "bench_module", os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)
ClockSampler = bench.ClockSampler


def _line(t, sm, power_cap=False, thermal=False):
    lt = time.localtime(t)
    stamp = time.strftime("%Y/%m/%d %H:%M:%S", lt) + ".%03d" % int(round((t % 1) * 1000) % 1000)
    act = lambda on: "Active" if on else "Not Active"  # noqa: E731
    return (f"{stamp}, 0, {sm}, 1965, 812.5, 0x0000000000000004, Not Active, {act(thermal)}, Not Active, "
            f"{act(power_cap)}")


def test_parse_keeps_well_formed_samples():
    t = 1_700_000_000.25
    lines = [_line(t + 0.1 * i, 1900 + i) for i in range(4)] + ["", "garbage", "[N/A], 0, [N/A]"]
    s = ClockSampler.parse(lines)
    assert len(s) == 4
    assert abs(s[0][0] - t) < 2e-3 and s[3][1] == 1903.0 and s[0][2] == 1965.0


def test_window_selects_inside_samples_and_reasons():
    t = 1_700_000_000.0
    lines = [_line(t + 0.1 * i, 1800 + 10 * i, power_cap=(i == 4)) for i in range(12)]
    c = ClockSampler.summarize(ClockSampler.parse(lines), t + 0.25, t + 0.75)
    assert c["samples"] == 5  # 0.3 .. 0.7
    assert c["sm_mhz"] == 1850.0 and c["sm_max_mhz"] == 1965.0
    assert c["reasons"] == ["sw_power_cap"]


def test_short_window_takes_nearest_neighbours():
    t = 1_700_000_000.0
    lines = [_line(t + 0.1 * i, 1900 + i, thermal=(i == 3)) for i in range(8)]
    c = ClockSampler.summarize(ClockSampler.parse(lines), t + 0.21, t + 0.28)
    assert c["samples"] == 2 and c["sm_mhz"] == 1902.5
    assert c["reasons"] == ["hw_thermal_slowdown"]


def test_no_samples_near_the_window():
    t = 1_700_000_000.0
    s = ClockSampler.parse([_line(t, 1965)])
    assert ClockSampler.summarize(s, t + 5.0, t + 6.0) is None
