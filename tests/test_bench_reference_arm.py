"""The reference arm of bench.py (`--impl reference`) times the reference's
own CPU executable and must load nothing of this package: run in a fresh
interpreter on a small grid, it leaves no `pursuit_evasion_b200` module and
no libpe_b200.so in the process.  Its plain-Python CFL restatement equals
the library's `pe_relative_cfl_limit` (native_relative.cpp:76-81)."""

import json
import subprocess
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]

PROBE = r"""
import json, sys
from types import SimpleNamespace
sys.path.insert(0, {repo!r})
import bench
bench.GRID = dict(positions=17, headings=12, p_speeds=7, e_speeds=7, extent=4.0)
bench.run_reference_arm(SimpleNamespace(gpus=1, steps=1, warmup=0), 1, 0)
mods = sorted(m for m in sys.modules if m.startswith("pursuit_evasion_b200"))
maps = open("/proc/self/maps").read()
print(json.dumps({{"modules": mods, "so_loaded": "libpe_b200.so" in maps}}))
"""


def test_reference_arm_loads_nothing_of_the_package():
    out = subprocess.run([sys.executable, "-c", PROBE.format(repo=str(REPO))],
                         capture_output=True, text=True, timeout=300, cwd="/")
    assert out.returncode == 0, out.stderr
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    line, probe = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["workload"].startswith("relative5d_eno2_lf_rk2 RelativeGrid(17,12,7,7")
    assert probe == {"modules": [], "so_loaded": False}


def test_reference_cfl_restatement_equals_library():
    import bench
    from pursuit_evasion_b200.reversible.free_dp import RelativeGrid
    from pursuit_evasion_b200.reversible.relative_solver import cfl_limit

    assert bench.reference_cfl_dt() == cfl_limit(bench.a3_config(), RelativeGrid(**bench.GRID))
