"""bench.py's host pieces, without a GPU: the nvidia-smi clock sampler keeps
only the rows of the timed region and reports throttle reasons."""
import os
import stat
import sys
import time

from conftest import ROOT


def _fake_smi(tmp_path, row, delay):
    path = tmp_path / "nvidia-smi"
    path.write_text("#!/bin/bash\nsleep %s\nwhile true; do echo \"%s\"; sleep 0.05; done\n"
                    % (delay, row))
    path.chmod(path.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


def test_clock_sampler_waits_for_its_first_row(tmp_path, monkeypatch):
    d = _fake_smi(tmp_path, "1965, 1965, 700.0, Not Active, Not Active, Not Active, Active", 0.3)
    monkeypatch.setenv("PATH", d + os.pathsep + os.environ["PATH"])
    sys.path.insert(0, ROOT)
    import bench
    with bench.Clocks(0) as clk:
        assert clk.skip >= 1          # the sampler was running before the region
        time.sleep(0.3)
    s = clk.summary()
    assert s["samples"] >= 2
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    sys.path.insert(0, ROOT)
    import bench
    with bench.Clocks(0) as clk:
        pass
    assert clk.summary() == {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
