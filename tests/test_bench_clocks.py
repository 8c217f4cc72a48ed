"""bench.py's clock record: only samples taken inside the timed windows count,
a window shorter than the sampling interval still gets the sample that ends
it, and throttle reasons are read from the sampled rows.  A stand-in
nvidia-smi on PATH prints fixed rows, so no GPU is needed."""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _fake_smi(tmp_path, sm_mhz, cap_reason):
    exe = tmp_path / "nvidia-smi"
    cap = "Active" if cap_reason else "Not Active"
    exe.write_text("#!/bin/bash\nwhile true; do\n"
                   f'  echo "0, {sm_mhz}, 1965, 700.0, 0x4, Not Active, Not Active, '
                   f'Not Active, {cap}"\n'
                   "  sleep 0.05\ndone\n")
    exe.chmod(0o755)
    return str(tmp_path)


def _sampler(monkeypatch, tmp_path, sm_mhz=1965, cap_reason=False):
    monkeypatch.setenv("PATH", _fake_smi(tmp_path, sm_mhz, cap_reason) + os.pathsep +
                       os.environ["PATH"])
    sys.path.insert(0, ROOT)
    import bench
    return bench.ClockSampler(0)


def test_samples_only_inside_windows(monkeypatch, tmp_path):
    clk = _sampler(monkeypatch, tmp_path).__enter__()
    try:
        time.sleep(0.4)  # outside any window: not kept
        assert clk.rows == []
        with clk.window():
            time.sleep(0.3)
        n = len(clk.rows)
        assert n >= 2
        time.sleep(0.3)
        assert len(clk.rows) == n
        s = clk.summary()
        assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
        assert s["reasons"] == [] and s["samples"] == n
    finally:
        clk.__exit__()


def test_short_window_keeps_the_next_sample(monkeypatch, tmp_path):
    clk = _sampler(monkeypatch, tmp_path, sm_mhz=1200, cap_reason=True).__enter__()
    try:
        with clk.window():
            pass  # far shorter than the 50 ms interval
        s = clk.summary()
        assert s["samples"] >= 1
        assert s["sm_mhz"] == 1200.0 and s["reasons"] == ["sw_power_cap"]
    finally:
        clk.__exit__()


def test_no_sampler_reports_unsampled(monkeypatch, tmp_path):
    monkeypatch.setenv("PATH", str(tmp_path))  # no nvidia-smi at all
    sys.path.insert(0, ROOT)
    import bench
    with bench.ClockSampler(0) as clk, clk.window():
        pass
    assert clk.summary()["reasons"] == ["unsampled"]
