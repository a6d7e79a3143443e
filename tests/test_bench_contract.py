"""The reference arm of bench.py (the FP64 oracle timed on the host cores)
prints the same metric line as the GPU arm, over every slice of the
workload, without a GPU and without loading any library of the product."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_the_contract_line():
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2',"
            " '--warmup', '1', '--nslice', '6']; runpy.run_path('bench.py', run_name='__main__');"
            " maps = open('/proc/self/maps').read();"
            " print('MAPS', 'libg4b200' in maps, 'libg4host' in maps, 'libg4oracle' in maps)")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    sys.path.insert(0, str(ROOT))
    import bench
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("time-dependent SASE 6 slices x 8192")
    assert d["config"]["nslice"] == 6
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "all 6 slices per step, 2 of 2 timed steps" in cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    maps = [l for l in out.stdout.splitlines() if l.startswith("MAPS")]
    assert maps == ["MAPS False False True"], maps
