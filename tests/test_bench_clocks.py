"""The benchmark's clock record: how samples become the `clocks` object of the JSON line.

On a GPU box the sampler reads NVML in a thread of the bench process (nvidia-smi
as the fallback).  These tests plant samples of both kinds and check the
summary the line carries: median SM clock, maximum clock, the throttle reasons
seen in any sample, median power.  Without a GPU the sampler must stay silent.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_nvml_samples_summary():
    c = bench.ClockSampler(0)
    c.source = "nvml"
    # (SM MHz, max SM MHz, power W, NVML clocks-event reason bits)
    c.samples = [(1965.0, 1965.0, 500.0, 0), (1890.0, 1965.0, 990.0, 0x4), (1965.0, 1965.0, 620.0, 0)]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert s["power_w"] == 620.0 and s["samples"] == 3 and s["source"] == "nvml"


def test_nvml_reason_bits_map_to_names():
    c = bench.ClockSampler(0)
    c.samples = [(1500.0, 1965.0, 700.0, 0x8 | 0x40), (1400.0, 1965.0, 700.0, 0x20)]
    assert c.summary()["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]


def test_nvidia_smi_csv_summary(tmp_path):
    path = tmp_path / "clocks.csv"
    path.write_text("1965, 1965, 512.30, Not Active, Not Active, Not Active, Not Active\n"
                    "1837, 1965, 1005.64, Not Active, Not Active, Not Active, Active\n"
                    "1965, 1965, [N/A], Not Active, Not Active, Not Active, Not Active\n"
                    "garbage line\n")
    c = bench.ClockSampler(0)
    c.source = "nvidia-smi"
    c.path = str(path)
    s = c.summary()
    assert s["samples"] == 3 and s["sm_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert abs(s["power_w"] - 758.97) < 1e-9   # median of the two readable power values
    assert not os.path.exists(path)             # the temporary file is consumed


def test_sampler_without_gpu_is_silent():
    """No NVML device and no nvidia-smi here: entering and leaving raise nothing."""
    import torch
    if torch.cuda.is_available():
        return
    with bench.ClockSampler(0) as c:
        pass
    s = c.summary()
    assert s is None or s["samples"] >= 1
