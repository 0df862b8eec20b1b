"""bench.py's clock sampler against a stand-in nvidia-smi (CPU).

The stand-in prints a CSV sample every 50 ms in nvidia-smi's query format: SM
clock 1965 MHz with sw_power_cap active while a marker file exists (the
"load"), 300 MHz idle otherwise. Only the samples between mark_begin and
mark_end may be summarised.
"""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402

FAKE = r'''#!{python}
import os, sys, time
marker = {marker!r}
while True:
    busy = os.path.exists(marker)
    sm = 1965 if busy else 300
    cap = "Active" if busy else "Not Active"
    sys.stdout.write(f"0, {{sm}}, 1965, 500.00, 0x4, Not Active, Not Active, Not Active, {{cap}}\n")
    sys.stdout.flush()
    time.sleep(0.05)
'''


def _install_fake(tmp_path, monkeypatch):
    marker = tmp_path / "busy"
    exe = tmp_path / "nvidia-smi"
    exe.write_text(FAKE.format(python=sys.executable, marker=str(marker)))
    exe.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}{os.pathsep}{os.environ['PATH']}")
    return marker


def test_only_samples_under_load_are_summarised(tmp_path, monkeypatch):
    marker = _install_fake(tmp_path, monkeypatch)
    s = bench.ClockSampler(0)
    s.start()
    s.wait_ready()
    time.sleep(0.3)  # idle samples before the load
    marker.touch()
    time.sleep(0.12)  # the stand-in sees the marker on its next sample
    s.mark_begin()
    time.sleep(0.5)
    s.mark_end()
    marker.unlink()
    time.sleep(0.3)  # idle samples after the load
    r = s.stop()
    assert r["sm_mhz"] == 1965.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]
    assert r["samples_under_load"] >= 5 and r["samples"] == r["samples_under_load"]
    assert r["interval_ms"] == 50


def test_without_nvidia_smi(monkeypatch, tmp_path):
    monkeypatch.setenv("PATH", str(tmp_path))  # nothing to run
    s = bench.ClockSampler(0)
    s.start()
    s.wait_ready(timeout=0.2)
    s.mark_begin()
    s.mark_end()
    assert s.stop()["reasons"] == ["nvidia-smi unavailable"]
