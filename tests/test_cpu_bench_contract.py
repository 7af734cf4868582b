"""The JSON line of `bench.py --impl reference` (CPU only).

That arm times the CPU restatement of the walk on the host cores and must
print one JSON line with the same metric, unit and workload as the GPU arm,
plus its `cpu_baseline` and a zero-copy `e2e` block.  Under a multi-rank
launch only rank 0 runs; the other ranks exit 0 without output.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _run(extra_env=None):
    env = dict(os.environ)
    env.pop("RANK", None)
    env.pop("WORLD_SIZE", None)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "0"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_json_line():
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, p.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "photons/s"
    assert d["higher_is_better"] is True
    assert d["config"]["workload"] == bench.WORKLOAD
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


@pytest.mark.parametrize("rank", ["1", "3"])
def test_reference_arm_other_ranks_print_nothing(rank):
    p = _run({"RANK": rank, "WORLD_SIZE": "4"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_reference_arm_loads_only_the_oracle():
    """`bench.py --impl reference` times the CPU restatement; it must not
    import this library's Python package nor map its shared library (it
    reads the configuration with the oracle's own reader)."""
    import subprocess
    import sys
    code = (
        "import runpy, sys\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0',"
        " '--ref-sample', '2000']\n"
        "try:\n    runpy.run_path('bench.py', run_name='__main__')\n"
        "except SystemExit:\n    pass\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('PRODUCT', 'libmcml_b200' in maps, 'mcml_gpu_b200' in sys.modules)\n"
        "print('ORACLE', 'liboracle' in maps)\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    assert "PRODUCT False False" in r.stdout, r.stdout
    assert "ORACLE True" in r.stdout, r.stdout
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][0]
    assert '"impl": "reference"' in line
