"""bench.py's clock sampler against a stand-in `nvidia-smi` (a shell script
on PATH that prints the queried CSV fields every 50 ms): the samples inside a
short timed window are kept, throttle reasons are reported, and a window
shorter than the sampling interval still gets the nearest sample."""
import importlib.util
import os
import stat
import time

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _fake_smi(tmp_path, power_cap: str):
    path = tmp_path / "nvidia-smi"
    path.write_text("#!/bin/bash\nsleep 0.2\nwhile true; do\n"
                    f"  echo \"0, 1965, 1965, 900.0, 0x4, Not Active, Not Active, Not Active, {power_cap}\"\n"
                    "  sleep 0.05\ndone\n")
    path.chmod(path.stat().st_mode | stat.S_IEXEC)


def test_samples_inside_the_window_with_reasons(tmp_path, monkeypatch):
    _fake_smi(tmp_path, "Active")
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ['PATH']}")
    b = _bench()
    c = b.ClockSampler(0)
    c.start()
    t0 = time.perf_counter()
    time.sleep(0.5)
    clk = c.stop(t0, time.perf_counter())
    assert clk["samples"] >= 5
    assert clk["sm_mhz"] == 1965.0 and clk["sm_max_mhz"] == 1965.0
    assert clk["reasons"] == ["sw_power_cap"]


def test_short_window_gets_the_nearest_sample(tmp_path, monkeypatch):
    _fake_smi(tmp_path, "Not Active")
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ['PATH']}")
    b = _bench()
    c = b.ClockSampler(0)
    c.start()
    t0 = time.perf_counter()
    time.sleep(0.01)
    clk = c.stop(t0, time.perf_counter())
    assert clk["samples"] >= 1 and clk["reasons"] == []


def test_no_nvidia_smi_gives_none(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))       # an empty directory: nothing to run
    b = _bench()
    c = b.ClockSampler(0)
    c.start()
    assert c.stop(0.0, 1.0) is None
