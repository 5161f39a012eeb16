"""bench.py's clock sampler on a machine without a GPU: it reads nothing,
reports no clocks, and leaves the interpreter's GIL switch interval as it
found it (the sampler shortens it only for the timed region)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_clock_sampler_without_gpu_restores_switch_interval():
    sys.path.insert(0, ROOT)
    import bench
    before = sys.getswitchinterval()
    c = bench.ClockSampler(0)
    c.start()
    assert sys.getswitchinterval() <= 0.0002 + 1e-9
    out = c.stop()
    assert sys.getswitchinterval() == before
    # No NVML device and no nvidia-smi here: nothing sampled, nothing claimed.
    assert out is None or out["samples"] >= 1


def test_clock_sampler_parses_nvidia_smi_lines():
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler(0)
    c.proc = type("P", (), {"terminate": lambda self: None, "wait": lambda self, timeout: 0})()
    c.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Active",
               "0, 1950, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "garbage"]
    out = c.stop()
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"],
                   "samples": 2, "source": "nvidia-smi"}
