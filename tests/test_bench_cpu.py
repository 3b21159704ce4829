"""Host logic of bench.py that needs no GPU: the clock record read from
nvidia-smi's CSV lines (median SM clock, throttle reasons seen while the
timed region ran), which decides whether a bench line is kept."""
import sys

from conftest import ROOT


class _FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def _sampler(lines):
    sys.path.insert(0, ROOT)
    import bench
    s = bench.ClockSampler(0)
    s.proc = _FakeProc()
    s.lines = list(lines)
    return s


def test_clock_record_median_and_reasons():
    # index, clocks.sm, clocks.max.sm, power.draw, active mask, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    lines = [
        "0, 1965, 1965, 610.2, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1320, 1965, 998.6, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 702.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    rec = _sampler(lines).stop()
    assert rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["samples"] == 3                  # the malformed lines are skipped
    assert rec["reasons"] == ["sw_power_cap"]   # kept and noted, not a rejection reason


def test_clock_record_reports_thermal_slowdown():
    lines = ["0, 1500, 1965, 900.0, 0x0000000000000040, Not Active, Active, Not Active, Not Active"] * 3
    rec = _sampler(lines).stop()
    assert rec["reasons"] == ["hw_thermal_slowdown"] and rec["sm_mhz"] == 1500.0


def test_clock_record_without_nvidia_smi():
    sys.path.insert(0, ROOT)
    import bench
    s = bench.ClockSampler(0)  # never started: no process
    rec = s.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]
