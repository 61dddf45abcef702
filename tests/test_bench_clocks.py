"""bench.py's clock sampler against a stand-in nvidia-smi (no GPU): it waits for the sampler's first line before the
timed region, keeps only the samples printed after mark(), and reports the throttle reasons seen as Active."""
import os
import stat
import sys
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# one sample before the timed region at a low clock, then samples at the full clock with the power cap active
FAKE = """#!/bin/sh
echo "0, 1000, 1965, 300.0, 0x0, Not Active, Not Active, Not Active, Not Active"
sleep 0.3
while true; do
  echo "0, 1965, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active"
  sleep 0.05
done
"""


@pytest.fixture()
def fake_smi(tmp_path, monkeypatch):
    path = tmp_path / "nvidia-smi"
    path.write_text(FAKE)
    path.chmod(path.stat().st_mode | stat.S_IXUSR)
    monkeypatch.setenv("PATH", str(tmp_path) + os.pathsep + os.environ.get("PATH", ""))
    return path


def test_clock_sampler_keeps_the_timed_region(fake_smi):
    sys.path.insert(0, ROOT)
    import bench
    clocks = bench.Clocks(0)
    clocks.mark()  # the low-clock line printed before this point belongs to no timed step
    time.sleep(0.8)
    got = clocks.stop()
    assert got["samples"] >= 3, got
    assert got["sm_mhz"] == 1965.0 and got["sm_max_mhz"] == 1965.0, got
    assert got["reasons"] == ["sw_power_cap"], got


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    sys.path.insert(0, ROOT)
    import bench
    clocks = bench.Clocks(0)
    clocks.mark()
    got = clocks.stop()
    assert got["sm_mhz"] is None and got["reasons"] == ["nvidia-smi unavailable"]
