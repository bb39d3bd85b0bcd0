"""bench.py's clock record during the timed region: the in-process NVML
sampler (reading only) merged with nvidia-smi's samples, exercised on the CPU
against a fake NVML module."""
import sys
import time
import types

import pytest


def _fake_nvml(mhz=1965, reasons=0x4):
    nv = types.ModuleType("pynvml")
    nv.NVML_CLOCK_SM = 1
    nv.nvmlClocksEventReasonHwSlowdown = 0x8
    nv.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    nv.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    nv.nvmlClocksEventReasonSwPowerCap = 0x4
    nv.calls = {"init": 0, "shutdown": 0}
    nv.nvmlInit = lambda: nv.calls.__setitem__("init", nv.calls["init"] + 1)
    nv.nvmlShutdown = lambda: nv.calls.__setitem__("shutdown", nv.calls["shutdown"] + 1)
    nv.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    nv.nvmlDeviceGetHandleByUUID = lambda u: ("gpu", u)
    nv.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965
    nv.nvmlDeviceGetClockInfo = lambda h, c: mhz
    nv.nvmlDeviceGetCurrentClocksEventReasons = lambda h: reasons
    return nv


@pytest.fixture
def bench_mod(monkeypatch):
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    monkeypatch.syspath_prepend(root)
    import bench
    return bench


def test_nvml_samples_fill_the_record(bench_mod, monkeypatch):
    nv = _fake_nvml(mhz=1900, reasons=0x4 | 0x20)
    monkeypatch.setitem(sys.modules, "pynvml", nv)
    monkeypatch.setenv("PATH", "")  # no nvidia-smi: NVML alone
    c = bench_mod.Clocks(0)
    time.sleep(0.06)
    rec = c.stop()
    assert rec is not None and rec["samples_nvml"] >= 3 and rec["samples_nvidia_smi"] == 0
    assert rec["sm_mhz"] == 1900.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]
    assert nv.calls == {"init": 1, "shutdown": 1}


def test_no_nvml_no_smi_gives_no_record(bench_mod, monkeypatch):
    broken = types.ModuleType("pynvml")

    def fail():
        raise RuntimeError("no driver")
    broken.nvmlInit = fail
    monkeypatch.setitem(sys.modules, "pynvml", broken)
    monkeypatch.setenv("PATH", "")
    c = bench_mod.Clocks(0)
    assert c.stop() is None


def test_visible_devices_map_to_physical(bench_mod, monkeypatch):
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "3,5")
    assert bench_mod._physical_gpu(1) == "5"
    monkeypatch.delenv("CUDA_VISIBLE_DEVICES")
    assert bench_mod._physical_gpu(2) == "2"
