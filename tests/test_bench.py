"""bench.py's reference arm on CPU: the JSON line it prints (metric, unit,
cpu_baseline, e2e with no host-device bytes) and the rule that under a
multi-rank launch only rank 0 runs it."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from oracle import py_oracle

ROOT = Path(__file__).resolve().parent.parent
pytestmark = pytest.mark.skipif(not py_oracle.ref_available("timed"),
                                reason="the reference library is not built")


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                           "--workload", "su2_16", "--steps", "1", "--warmup", "3"],
                          capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)


def test_reference_arm_json_line():
    p = _run({"OMP_NUM_THREADS": "2"})
    assert p.returncode == 0, p.stderr
    lines = [x for x in p.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "smeared+measured sites/s" and d["unit"] == "sites/s"
    assert d["value"] > 0 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "su2_16" and d["config"]["sites"] == 16 ** 4
    # the same config dict as the GPU arm's line
    import bench
    assert d["config"] == bench.config_dict("su2_16", bench.WORKLOADS["su2_16"], 1)
    assert set(d["phase_seconds"]) == {"hyp", "ape", "wilson"}
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "reference" and cb["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "sites/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_do_no_work():
    p = _run({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_reference_arm_loads_no_product_library():
    """The reference arm builds its input with the checkers' copy of the
    generator (oracle/libgen.so): the process maps no product library."""
    code = (
        "import runpy, sys\n"
        f"sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'su2_16', "
        f"'--steps', '1', '--warmup', '3']\n"
        "try:\n"
        f"    runpy.run_path({str(ROOT / 'bench.py')!r}, run_name='__main__')\n"
        "except SystemExit as e:\n"
        "    assert not e.code, e.code\n"
        "maps = open('/proc/self/maps').read()\n"
        "assert 'libgc_b200' not in maps, 'product library mapped'\n"
        "assert 'general_code_b200' not in sys.modules\n"
        "assert 'libgen.so' in maps\n"
        "print('CLEAN')\n")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=300, cwd=ROOT, env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip().endswith("CLEAN")
