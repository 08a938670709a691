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


def test_reference_arm_builds_the_workload_without_this_library(tmp_path):
    """The reference arm builds the benchmarked plan from the package's
    host-side classes: libpb_b200.so must not be mapped in that process, and
    both arms print the same `config` object."""
    import subprocess
    code = (
        "import sys, json; sys.path.insert(0, %r); import bench\n"
        "c = bench.plan_case(3)\n"
        "cfg = bench.plan_config(c, 'forward')\n"
        "h2d, d2h = bench.reference_copy_bytes(c)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'cfg': cfg, 'lib': 'libpb_b200' in maps, 'h2d': h2d, 'd2h': d2h,\n"
        "                  'mods': sorted(m for m in sys.modules if m.startswith('dosecuda_b200'))}))\n"
    ) % ROOT
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=300, check=True).stdout
    import json
    r = json.loads(out.strip().splitlines()[-1])
    assert r["lib"] is False
    assert "dosecuda_b200._lib" not in r["mods"] and "dosecuda_b200.engine" not in r["mods"]
    cfg = r["cfg"]
    assert cfg["voxels"] == 256 * 256 * 160 and cfg["beams"] == 4 and cfg["mode"] == "forward"
    assert 18000 <= cfg["spots"] <= 21000
    V = cfg["voxels"]
    # per beam: RLSP up twice and WET up once; WET and dose back
    assert r["h2d"] >= 4 * 12 * V
    assert r["d2h"] == 4 * 8 * V


def test_reference_arm_prints_unavailable_for_modes_it_lacks():
    import json
    import subprocess
    for extra in (["--mode", "grad"], ["--workload", "batch"], ["--workload", "optimize"]):
        out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                              "reference"] + extra, capture_output=True, text=True, timeout=120,
                             check=True).stdout
        line = json.loads(out.strip().splitlines()[-1])
        assert line["impl"] == "reference" and "unavailable" in line
