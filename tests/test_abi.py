"""The C ABI library loads and exports every entry point include/voila_cuda.h declares;
host-only entry points behave; without a GPU the device entry points fail cleanly."""
import os
import re
import subprocess

import numpy as np
import pytest

from vldb_voila_b200 import engine as E

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "voila_cuda.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:const char\*|int)\s+(vc_\w+)\(", text, re.M)))


def test_every_declared_symbol_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", E.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (vc_\w+)", out))
    missing = [s for s in declared() if s not in exported]
    assert not missing, missing
    assert len(declared()) >= 30


def test_library_loads_and_reports_version():
    assert b"sm_100a" in E.lib().vc_version()


def test_no_device_is_a_clean_error():
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a GPU is present")
    with pytest.raises(E.VoilaError) as ex:
        E.Engine(0)
    assert ex.value.code == 7


def test_workload_description_and_host_generator():
    w = E.workload("join_aggr:build=1000,probe=5000,sel=0.3,seed=4")
    assert w.template == "join_aggr" and w.tables == {"orders": 1000, "lineitem": 5000}
    keys = E.generate_host([c for c in w.columns if c.name == "o_orderkey"][0])
    assert sorted(keys.tolist()) == list(range(1, 1001))  # a permutation of 1..n
    attr = E.generate_host([c for c in w.columns if c.name == "o_attr"][0])
    assert attr.min() >= 0 and attr.max() <= 9999
    with pytest.raises(E.VoilaError):
        E.workload("nosuch:rows=1")


def test_zipf_generator_is_skewed():
    w = E.workload("groupby:rows=200000,keys=1000,zipf=1.25,seed=3")
    col = [c for c in w.columns if c.name == "l_orderkey"][0]
    k = E.generate_host(col)
    counts = np.bincount(k, minlength=1001)
    assert k.min() >= 1 and k.max() <= 1000
    # P(1)/P(2) = 2^1.25 for Zipf(1.25)
    assert 2.0 < counts[1] / counts[2] < 2.8


def test_batch_specs_are_seeded():
    a = E.batch_specs(16, 5)
    assert a == E.batch_specs(16, 5) and a != E.batch_specs(16, 6)
    assert {s.split(":")[0] for s in a} <= {"sel_aggr", "join_aggr", "groupby"}


def test_reference_side_glue_library_exports_the_generated_query_abi():
    """The CUDA flavor's generated library (oracle/ref/cuda_glue.inc, built for each golden
    case by oracle/ref/build_queries.py) exports the reference's voila_query_* ABI and, driven
    by the reference's runner on a host without a GPU, fails with the engine's message instead
    of crashing."""
    import os
    import subprocess
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    rdir = os.path.join(repo, "oracle", "_ref", "avx512")
    lib = os.path.join(rdir, "q_golden_join_n_cuda.so")
    with open("/proc/cpuinfo") as f:
        avx512 = "avx512f" in f.read()
    if not os.path.exists(lib) or not avx512:
        pytest.skip("the reference build in oracle/_ref is not available here")
    syms = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    for s in ("voila_query_new", "voila_query_run", "voila_query_reset", "voila_query_free"):
        assert f" T {s}" in syms
    import torch
    if torch.cuda.is_available():
        return
    r = subprocess.run([os.path.join(rdir, "ref_run"), "--workload", "star:rows=1000,custs=50", "--lib", lib,
                        "--flavor", "cuda", "--reps", "1"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "cuda flavor:" in r.stderr


def test_product_code_never_reaches_the_oracle():
    """The library and its Python binding import, link or run nothing under oracle/ (the oracle
    is test infrastructure: only tests, smoke() and bench.py's baseline legs use it)."""
    import ast
    import os
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vldb_voila_b200")
    for name in os.listdir(pkg):
        if name.endswith(".py"):
            tree = ast.parse(open(os.path.join(pkg, name)).read())
            for node in ast.walk(tree):
                if isinstance(node, ast.Import):
                    assert not any(a.name.split(".")[0] == "oracle" for a in node.names), name
                elif isinstance(node, ast.ImportFrom):
                    assert (node.module or "").split(".")[0] != "oracle", name
    csrc = os.path.join(pkg, "csrc")
    for root, _, files in os.walk(csrc):
        for name in files:
            if name.endswith((".cpp", ".hpp", ".cu", ".cuh", ".h")):
                text = open(os.path.join(root, name)).read()
                assert "oracle/" not in text and "voila_oracle" not in text, name
