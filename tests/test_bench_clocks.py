"""bench.py's clock sampler on CPU against a fake NVML: the SM clock median,
the maximum clock and the clock-event reasons seen during the sampled region,
read through the read-only NVML queries the sampler uses."""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class FakeNvml:
    NVML_CLOCK_SM = 1

    def __init__(self, clocks, bits):
        self.clocks, self.bits, self.i = clocks, bits, 0
        self.inited = self.shut = False

    def nvmlInit(self):
        self.inited = True

    def nvmlShutdown(self):
        self.shut = True

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("gpu", i)

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        assert kind == self.NVML_CLOCK_SM
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        assert kind == self.NVML_CLOCK_SM
        v = self.clocks[min(self.i, len(self.clocks) - 1)]
        return v

    def nvmlDeviceGetCurrentClocksThrottleReasons(self, h):
        v = self.bits[min(self.i, len(self.bits) - 1)]
        self.i += 1
        return v


def test_nvml_samples_median_and_reasons():
    sys.path.insert(0, ROOT)
    import bench
    nv = FakeNvml([1965, 1950, 1965, 1965, 1320], [0, 0x4, 0x4, 0, 0x4])
    with bench.ClockSampler(0, period=0.005, nvml=nv) as clk:
        time.sleep(0.1)
    s = clk.summary()
    assert nv.inited and nv.shut
    assert s["samples"] >= 5
    assert s["sm_max_mhz"] == 1965.0
    assert s["sm_mhz"] == 1320.0 or s["sm_mhz"] >= 1950.0
    assert s["reasons"] == ["sw_power_cap"]


def test_thermal_and_hw_slowdown_bits_are_reported():
    sys.path.insert(0, ROOT)
    import bench
    nv = FakeNvml([1500], [0x8 | 0x40 | 0x20])
    with bench.ClockSampler(0, period=0.005, nvml=nv) as clk:
        time.sleep(0.03)
    assert clk.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_short_region_still_has_a_sample():
    sys.path.insert(0, ROOT)
    import bench
    nv = FakeNvml([1965], [0])
    with bench.ClockSampler(0, period=10.0, nvml=nv) as clk:
        pass
    assert clk.summary()["samples"] == 1
