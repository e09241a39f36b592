"""Host-side pieces of bench.py that decide how a bench line is read: the clock and throttle
summary taken from nvidia-smi samples during the timed region."""
import importlib.util
import os

ROOT = os.path.join(os.path.dirname(__file__), "..")


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def _sampler(tmp_path, lines):
    bench = _bench()
    s = bench.ClockSampler(0)
    s.path = str(tmp_path / "clocks.csv")
    s.proc = object()  # samples were taken
    with open(s.path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return s


def test_clock_summary_takes_median_max_and_active_reasons(tmp_path):
    rows = [
        "0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1800, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 1950, 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "garbage line",
        "0, [N/A], 1965, 950.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ]
    summary = _sampler(tmp_path, rows).summary()
    assert summary == {"sm_mhz": 1950.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}


def test_clock_summary_reports_throttling_and_missing_samples(tmp_path):
    rows = ["0, 1200, 1965, 500.0, 0x8, Active, Not Active, Active, Not Active"]
    assert _sampler(tmp_path, rows).summary()["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert _sampler(tmp_path, ["no samples here"]).summary()["reasons"] == ["unsampled"]
    bench = _bench()
    assert bench.ClockSampler(0).summary()["reasons"] == ["unsampled"]  # nvidia-smi never started
