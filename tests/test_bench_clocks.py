"""bench.py's clock sampler on CPU, against a stand-in nvidia-smi that
prints a query line every 20 ms: the sampler waits for its first line
before the timed region, keeps the lines from mark() on plus the first one
after stop(), and reports the median SM clock and the active throttle
reasons."""
import os
import stat
import time

import bench


def _fake_smi(tmp_path, line):
    exe = tmp_path / "nvidia-smi"
    exe.write_text("#!/bin/sh\nwhile true; do echo '%s'; sleep 0.02; done\n" % line)
    exe.chmod(exe.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


def test_clock_sampler_reads_samples_and_reasons(tmp_path, monkeypatch):
    d = _fake_smi(tmp_path, "0, 1800, 1965, 700.5, 0x4, Not Active, Not Active, Not Active, Active")
    monkeypatch.setenv("PATH", d + os.pathsep + os.environ["PATH"])
    c = bench.ClockSampler(0)
    c.start()
    c.mark()
    time.sleep(0.1)
    r = c.stop()
    assert r is not None
    assert r["sm_mhz"] == 1800.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]
    assert r["samples"] >= 2


def test_clock_sampler_short_region_keeps_one_sample(tmp_path, monkeypatch):
    d = _fake_smi(tmp_path, "0, 1965, 1965, 500.0, 0x0, Not Active, Not Active, Not Active, Not Active")
    monkeypatch.setenv("PATH", d + os.pathsep + os.environ["PATH"])
    c = bench.ClockSampler(0)
    c.start()
    c.mark()
    r = c.stop()  # no time in between: the first sample after stop() is kept
    assert r is not None and r["samples"] >= 1 and r["reasons"] == []


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    c = bench.ClockSampler(0)
    c.start()
    c.mark()
    assert c.stop() is None
