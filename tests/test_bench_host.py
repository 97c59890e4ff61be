"""Host logic of bench.py on the CPU: the DRAM-traffic lookup (exact and
scaled from a smaller capture) and the parsing of the NVML clock samples."""
import importlib.util
import os

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(REPO, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_traffic_lookup(bench):
    exact = bench.read_traffic("int8_tc_modular_x2_n4096")
    assert exact == 1489598464.0
    # a size above the largest capture scales by (n / n0)^2
    assert bench.read_traffic("int8_tc_modular_x2_n8192", scale_from_smaller=True) == 4 * exact
    assert bench.read_traffic("int8_tc_modular_x2_n8192") is None
    assert bench.read_traffic("no_such_kernel_n8192", scale_from_smaller=True) is None


class _Proc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


class _Thread:
    def join(self, timeout=None):
        pass


def test_nvml_sample_parsing(bench):
    s = bench.NvmlClockSampler(0)
    s.proc, s.thread, s.max_mhz = _Proc(), _Thread(), 1965.0
    s.lines = ["1965 0\n", "1900 4\n", "1965 1\n", "garbage\n"]
    out = s.stop()
    assert out["samples"] == 3 and out["sm_mhz"] == 1965.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]
    s.lines = ["1300 72\n"]  # hw_slowdown (8) + hw_thermal (64)
    out = s.stop()
    assert out["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
