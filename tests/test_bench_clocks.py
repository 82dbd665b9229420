"""The benchmark's clock sampler on the host, against a stand-in
``nvidia-smi`` that prints one CSV sample every 100 ms: a timed region
shorter than the sampling period still reports one sample (the first one
after the region, marked as such), a longer one reports the samples inside
it, and active throttle reasons are collected."""

import importlib.util
import os
import stat
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

FAKE = """#!/bin/sh
while true; do
  echo "0, 1965, 1965, 512.0, 0x0000000000000004, Not Active, Not Active, Not Active, Active"
  sleep 0.1
done
"""


def _bench():
    spec = importlib.util.spec_from_file_location("bench_for_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["bench_for_test"] = mod
    spec.loader.exec_module(mod)
    return mod


def _fake_smi(tmp_path, monkeypatch):
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE)
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ.get('PATH', '')}")


def test_short_region_takes_the_next_sample(tmp_path, monkeypatch):
    _fake_smi(tmp_path, monkeypatch)
    b = _bench()
    with b.ClockSampler(0) as c:
        time.sleep(0.005)
    s = c.summary()
    assert s["samples"] >= 1 and s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    assert "window" in s


def test_long_region_reports_its_own_samples(tmp_path, monkeypatch):
    _fake_smi(tmp_path, monkeypatch)
    b = _bench()
    with b.ClockSampler(0) as c:
        time.sleep(0.45)
    s = c.summary()
    assert s["samples"] >= 3
    assert "window" not in s


def test_no_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    b = _bench()
    with b.ClockSampler(0) as c:
        pass
    s = c.summary()
    assert s["sm_mhz"] is None
