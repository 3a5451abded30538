"""Host logic of bench.py (no GPU): the clock sampler against a fake NVML,
and its fallback when NVML does not load."""
import importlib.util
import os
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class FakeNVML:
    """The read-only NVML calls the sampler makes, with scripted answers."""
    NVML_CLOCK_SM = 1
    nvmlClocksThrottleReasonSwPowerCap = 0x4
    nvmlClocksThrottleReasonHwSlowdown = 0x8
    nvmlClocksThrottleReasonSwThermalSlowdown = 0x20
    nvmlClocksThrottleReasonHwThermalSlowdown = 0x40

    def __init__(self, clocks, reasons, fail_init=False):
        self.clocks, self.reasons, self.fail_init = list(clocks), list(reasons), fail_init
        self.calls, self.shutdown = 0, False

    def nvmlInit(self):
        if self.fail_init:
            raise RuntimeError("no NVML")

    def nvmlShutdown(self):
        self.shutdown = True

    def nvmlDeviceGetHandleByIndex(self, i):
        assert i == 3
        return "h"

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        assert (h, kind) == ("h", 1)
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        self.calls += 1
        return self.clocks[min(self.calls - 1, len(self.clocks) - 1)]

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return self.reasons[min(self.calls, len(self.reasons) - 1)]

    def nvmlDeviceGetCurrentClocksThrottleReasons(self, h):
        raise AssertionError("the newer query answers, so the older one is not used")


class OlderNVML(FakeNVML):
    """A driver without the clocks-event query: the throttle-reasons name."""

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        raise RuntimeError("function not found")

    def nvmlDeviceGetCurrentClocksThrottleReasons(self, h):
        return 0x40


def test_clocks_from_nvml_median_and_reasons():
    b = _bench()
    fake = FakeNVML(clocks=[1965, 1965, 1950, 1965, 1965], reasons=[0, 0, 0x4, 0, 0x4 | 0x8])
    c = b.Clocks(3, nvml=fake)
    c.start()
    time.sleep(0.15)
    out = c.stop()
    assert out["source"] == "nvml"
    assert out["samples"] >= 5  # every 10 ms
    assert out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert fake.shutdown


def test_clocks_from_an_older_nvml():
    b = _bench()
    c = b.Clocks(3, nvml=OlderNVML(clocks=[1900], reasons=[0]))
    c.start()
    time.sleep(0.05)
    out = c.stop()
    assert out["source"] == "nvml" and out["reasons"] == ["hw_thermal_slowdown"]


def test_clocks_without_nvml_fall_back_to_nvidia_smi(monkeypatch):
    b = _bench()
    fake = FakeNVML(clocks=[1965], reasons=[0], fail_init=True)
    c = b.Clocks(3, nvml=fake)
    # an nvidia-smi that answers with one line of the queried fields
    monkeypatch.setattr(c, "_smi_read", lambda: (1800.0, 1965.0, ("sw_power_cap",)))
    c.start()
    time.sleep(0.05)
    out = c.stop()
    assert out["source"] == "nvidia-smi"
    assert out["samples"] >= 1
    assert out["sm_mhz"] == 1800.0 and out["reasons"] == ["sw_power_cap"]


def test_clocks_with_no_source_report_it():
    b = _bench()
    c = b.Clocks(3, nvml=FakeNVML(clocks=[1], reasons=[0], fail_init=True))
    c._smi_read = lambda: None
    c.start()
    time.sleep(0.02)
    out = c.stop()
    assert out["sm_mhz"] is None and out["reasons"] == ["nvidia-smi unavailable"]


def test_advect_pairs_of_the_metric_workload():
    """Bound sheet + 400 wake ring rows as sources; node rows 1..401 as targets
    of the first RK2 evaluation, rows 6..401 of the second."""
    b = _bench()
    segs = (33 * 128 + 32 * 129) + (401 * 128 + 400 * 129)
    assert b._heave_pitch().advect_pairs() == (401 + 396) * 129 * segs
