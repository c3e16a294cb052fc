"""bench.py's clock record (no GPU): the sampler polls NVML while the timed
steps run and reports the median SM clock under load and every throttle
reason seen, which is what decides whether a measurement is kept.  A fake NVML
and a fake CUDA event stand in for the device."""
import sys
import types

import pytest

import bench


class FakeEvent:
    """Completes after `n` queries, like an event recorded behind n polls' worth of work."""

    def __init__(self, n):
        self.n = n
        self.synced = False

    def query(self):
        self.n -= 1
        return self.n < 0

    def synchronize(self):
        self.synced = True


def fake_nvml(clocks, reasons):
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksEventReasonHwSlowdown = 0x8
    nv.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nv.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksEventReasonSwPowerCap = 0x4
    it = {"k": 0}
    nv.nvmlInit = lambda: None
    nv.nvmlShutdown = lambda: None
    nv.nvmlDeviceGetHandleByPciBusId = lambda bid: ("bus", bid)
    nv.nvmlDeviceGetHandleByIndex = lambda i: ("idx", i)
    nv.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965

    def clock(h, c):
        v = clocks[min(it["k"], len(clocks) - 1)]
        return v

    def reason(h):
        r = reasons[min(it["k"], len(reasons) - 1)]
        it["k"] += 1
        return r

    nv.nvmlDeviceGetClockInfo = clock
    nv.nvmlDeviceGetCurrentClocksEventReasons = reason
    return nv


@pytest.fixture
def nvml(monkeypatch):
    def install(clocks, reasons):
        monkeypatch.setitem(sys.modules, "pynvml", fake_nvml(clocks, reasons))
        import torch

        props = types.SimpleNamespace(pci_bus_id=0x18, pci_domain_id=0, pci_device_id=0)
        monkeypatch.setattr(torch.cuda, "get_device_properties", lambda i: props)

    return install


def test_samples_only_while_the_timed_steps_run(nvml):
    nvml([1965.0], [0])
    ev = FakeEvent(6)
    with bench.Clocks(0) as clk:
        clk.wait(ev)
    s = clk.summary()
    assert ev.synced
    assert s["source"] == "nvml" and s["samples"] == 6
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["reasons"] == []


def test_throttle_reasons_and_loaded_median(nvml):
    # one idle-looking sample (below half the peak) is left out of the median;
    # a power-cap sample and a thermal one are reported by name
    nvml([1965.0, 1900.0, 600.0, 1950.0, 1940.0], [0, 0x4, 0, 0x20, 0])
    with bench.Clocks(0) as clk:
        clk.wait(FakeEvent(5))
    s = clk.summary()
    assert s["samples"] == 5
    assert s["sm_mhz"] == pytest.approx(1945.0)
    assert s["reasons"] == ["sw_thermal_slowdown", "sw_power_cap"]


def test_no_nvml_reports_unsampled(monkeypatch):
    # without NVML the sampler falls back to nvidia-smi; with neither, the
    # record says so instead of inventing a clock
    monkeypatch.setitem(sys.modules, "pynvml", None)
    monkeypatch.setattr(bench.subprocess, "Popen", lambda *a, **k: (_ for _ in ()).throw(FileNotFoundError()))
    with bench.Clocks(0) as clk:
        clk.wait(FakeEvent(3))
    s = clk.summary()
    assert s["samples"] == 0 and s["reasons"] == ["unsampled"]
