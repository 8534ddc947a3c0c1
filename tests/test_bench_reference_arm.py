"""bench.py's reference arm on the CPU: it times the reference's own generated code (built from
the reference's sources into oracle/_ref) without importing this package, and prints the
contract's JSON line."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RDIR = os.path.join(REPO, "oracle", "_ref", "avx512")

RUN = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1", "--workload", "config2"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    assert e.code in (0, None), e.code
print("PACKAGE_IMPORTED", "vldb_voila_b200" in sys.modules)
"""


def _have_reference_build():
    if not os.path.exists(os.path.join(RDIR, "ref_run")):
        return False
    with open("/proc/cpuinfo") as f:
        return "avx512f" in f.read()


@pytest.mark.skipif(not _have_reference_build(), reason="needs the reference build (oracle/_ref) on an AVX-512 host")
def test_reference_arm_runs_only_the_reference():
    r = subprocess.run([sys.executable, "-c", RUN], cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["config"]["workload"].startswith("join_aggr:")
    assert line["unit"] == "fact rows/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "fact rows/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert "PACKAGE_IMPORTED False" in r.stdout
