"""bench.py's host logic without a GPU: the clock samples' summary (the
throttle reasons a run is judged by), the peak it reports against and the
workload description."""

import importlib.util
import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_clock_summary_reports_the_median_and_the_active_reasons():
    b = bench()
    c = b.Clocks(0)
    c.lines = [
        "0, 1965, 1965, 610.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0
    assert s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert s["samples"] == 3


def test_clock_summary_flags_thermal_and_hardware_slowdown():
    b = bench()
    c = b.Clocks(0)
    c.lines = ["0, 1200, 1965, 900, 0x48, Active, Not Active, Active, Not Active"]
    s = c.summary()
    assert s["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert s["sm_mhz"] == 1200.0


def test_clock_summary_without_samples():
    b = bench()
    s = b.Clocks(0).summary()
    assert s == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}


def test_peak_is_the_measured_copy_bandwidth_when_present():
    b = bench()
    value, kind = b.measured_peaks()
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path) and "hbm_gbs" in json.load(open(path)):
        assert kind == "measured"
        assert value == float(json.load(open(path))["hbm_gbs"])
    else:
        assert (value, kind) == (6650.0, "fallback")


def test_workload_description_names_the_configuration():
    b = bench()
    c = b.config(4194304, 65241322)
    assert c["workload"] == "rmat22-batched-bfs-1024-sources-caps-U1..16"
    assert c["nodes"] == 4194304 and c["edges"] == 65241322
    assert c["sources_per_rank"] == 1024
    # Both arms describe the same workload with the same keys: the GPU
    # arm's schedule is reported beside the config, not in it.
    assert set(c) == set(b.config(4194304, 65241322))
    assert "L2" in c["l2"]
    src, caps = b.sources_and_caps(4194304)
    assert len(src) == 1024 and src.max() < 4194304
    assert caps.min() >= 1 and caps.max() <= 16
    # Each rank draws its own sources (weak scaling).
    assert not (b.sources_and_caps(4194304, rank=1)[0] == src).all()
