"""The drop-in boundary exercised through the reference itself: for every golden case, the
reference's own runner (oracle/ref/ref_run: runtime::Database + QueryConfig + dlopen +
voila_query_new/reset/run/free, as Compiler::_run drives a generated library,
compiler.cpp:465-598) loads the CUDA flavor's generated library (oracle/ref/cuda_glue.inc
over libvoila_cuda.so, built by oracle/ref/build_queries.py) and its QueryResult rows must
equal the rows the reference's own vectorwise flavor produced for the same data."""
import os
import subprocess
import tempfile

import pytest

from helpers import golden_lines, manifest

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RDIR = os.path.join(REPO, "oracle", "_ref", "avx512")
CASES = sorted(manifest().items())


def _avx512():
    with open("/proc/cpuinfo") as f:
        return "avx512f" in f.read()


@pytest.mark.parametrize("name,entry", CASES, ids=[c[0] for c in CASES])
def test_reference_runner_drives_the_cuda_flavor(name, entry):
    lib = os.path.join(RDIR, f"q_golden_{name}_cuda.so")
    if not _avx512() or not os.path.exists(lib):
        pytest.skip("the reference's runner (AVX-512 build in oracle/_ref) is not available here")
    with tempfile.TemporaryDirectory() as tmp:
        res = os.path.join(tmp, "rows.txt")
        r = subprocess.run([os.path.join(RDIR, "ref_run"), "--workload", entry["spec"], "--lib", lib,
                            "--flavor", "cuda", "--threads", "1", "--reps", "2", "--result", res],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        got = sorted(l for l in open(res).read().split("\n") if l)
    assert got == golden_lines(name, "vectorwise")
