"""Host-side pieces of bench.py that decide whether a measurement stands (no GPU needed):
the clock record taken during the timed region and the default run length."""
import os
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _sampler_with(lines):
    s = bench.ClockSampler(0)
    fd, s.path = tempfile.mkstemp(suffix=".csv")
    with os.fdopen(fd, "w") as f:
        f.write("\n".join(lines) + "\n")
    return s


def test_clock_summary_median_max_and_reasons():
    na = "Not Active"
    lines = [
        f"0, 1965, 1965, 820.1, 0x0000000000000000, {na}, {na}, {na}, {na}",
        f"0, 1905, 1965, 990.4, 0x0000000000000004, {na}, {na}, {na}, Active",
        f"0, 1950, 1965, 870.0, 0x0000000000000000, {na}, {na}, {na}, {na}",
        "0, [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A]",     # unreadable sample
        "garbage",
    ]
    out = _sampler_with(lines).summary()
    assert out["samples"] == 3
    assert out["sm_mhz"] == 1950.0
    assert out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"]


def test_clock_summary_reports_slowdowns():
    na = "Not Active"
    lines = [f"0, 1400, 1965, 600.0, 0x0000000000000008, Active, {na}, Active, {na}"] * 4
    out = _sampler_with(lines).summary()
    assert out["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]
    assert out["sm_mhz"] == 1400.0


def test_clock_summary_without_samples():
    s = bench.ClockSampler(0)
    out = s.summary()
    assert out["sm_mhz"] is None and out["reasons"] == [] and out["samples"] == 0


def test_default_run_length(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.impl == "ours"
    assert a.warmup >= 3 and a.steps >= 1


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 runs the reference arm; the other ranks print nothing."""
    import subprocess
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""
