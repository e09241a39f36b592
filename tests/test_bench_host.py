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


def test_reference_arm_line_keeps_integer_steps_and_the_shared_config(monkeypatch):
    bench = _bench()
    monkeypatch.setattr(bench, "cpu_projection", lambda scene, tol, threads: (0.5, 53, "reference"))
    monkeypatch.setattr(bench, "scene_for", lambda size, rank: type("S", (), {"cells": size * size})())
    args = type("A", (), {"size": 64, "warmup": 1, "steps": 3, "gpus": 1, "tolerance": 1e-6})()
    line = bench.run_reference(args, 1, 0)
    assert line["steps"] == 3 and isinstance(line["steps"], int)
    # Both arms carry the same config: the same scene, stop rule and tolerance.
    assert line["config"] == bench.workload_config(64, 1e-6)
    assert line["iterations"] == 53
    assert bench.run_reference(args, 2, 1) is None  # other ranks do no work


def test_cuda_arm_never_overwrites_the_step_count():
    """`steps` is the timed step count; every leg sits under its own key."""
    import ast

    tree = ast.parse(open(os.path.join(ROOT, "bench.py")).read())
    writes = [n for n in ast.walk(tree) if isinstance(n, ast.Assign)
              for t in n.targets if isinstance(t, ast.Subscript) and isinstance(t.slice, ast.Constant)
              and t.slice.value == "steps"]
    assert writes == []
    src = open(os.path.join(ROOT, "bench.py")).read()
    assert 'line["step_leg"] = steps_measure(' in src


def test_gpus_flag_spawns_ranks_or_rejects_a_mismatch(monkeypatch):
    bench = _bench()
    calls = []
    monkeypatch.setattr(bench.subprocess, "call", lambda cmd: calls.append(cmd) or 0)
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.setattr(bench.sys, "argv", ["bench.py", "--gpus", "4", "--steps", "2"])
    try:
        bench.main()
    except SystemExit as e:
        assert e.code == 0
    assert len(calls) == 1
    cmd = calls[0]
    assert "torch.distributed.run" in cmd and "--nproc-per-node=4" in cmd and "127.0.0.1" in cmd
    assert cmd[-4:] == ["--gpus", "4", "--steps", "2"]
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(bench.sys, "argv", ["bench.py", "--gpus", "4"])
    try:
        bench.main()
        raise AssertionError("a world size that differs from --gpus must fail")
    except SystemExit as e:
        assert e.code == 2
