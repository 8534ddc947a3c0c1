"""Parity of the CUDA flavor (through the C ABI) with the reference and the oracle.

Bit-exact: result rows are compared as sorted QueryResult lines, like the reference's
Query::check_result (runtime_framework.cpp:220-280)."""
import numpy as np
import pytest

from helpers import golden_lines, manifest
from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, VoilaError, generate_workload_host, workload

pytestmark = pytest.mark.gpu

CASES = sorted(manifest().items())
FLAVORS = ["", "cuda(rows=8,threads=128,load=tma,stages=3)", "cuda(aggr=cache,cache=256,build=staged,compact=0)",
           "cuda(aggr=global,rows=1,threads=64,graph=0,prefetch=0,compact=-1)",
           "cuda(load=tma,build=staged,rows=2,lowcard=atomic)", "cuda(compact=0,lowcard=private,rows=8)",
           "cuda(hash=voila,lowcard=private,threads=128,fill=75)", "cuda(build=direct,prefetch=0)",
           "cuda(lowcard=redux,aggr=cache,cache=64)", "cuda(build=direct,probe=4,rows=2)",
           "cuda(build=staged,probe=32,compact=-1)", "cuda(aggr=part)",
           "cuda(aggr=part,parts=16,threads=128,rows=8,load=tma,stages=2)", "cuda(frows=1)",
           "cuda(frows=8,compact=0,threads=128,rows=2)", "cuda(lowcard=regs)",
           "cuda(lowcard=regs,load=tma,stages=2,rows=8,pgroups=2,threads=128)", "cuda(lowcard=regs,rows=1,prefetch=0)",
           "cuda(aggr=direct)", "cuda(aggr=dcache,cache=64,rows=8,threads=128)", "cuda(lowcard=combine)",
           "cuda(lowcard=packed,load=tma,stages=2,pgroups=3,rows=2)"]


def run_gpu(w, plan, flavor="", on_device=False, data=None):
    e = Engine(0)
    e.load_workload(w, data=data, on_device=on_device)
    q = e.query(plan, flavor)
    q.run()
    lines = q.result_lines()
    q.close()
    e.close()
    return lines


@pytest.mark.parametrize("flavor", FLAVORS)
@pytest.mark.parametrize("name,entry", CASES, ids=[c[0] for c in CASES])
def test_golden(name, entry, flavor):
    w = workload(entry["spec"])
    plan = entry["plan"] or w.plan
    assert run_gpu(w, plan, flavor) == golden_lines(name, "vectorwise")


FULL = [
    "sel_aggr:rows=6000000,seed=1",
    "join_aggr:build=1500000,probe=6000000,sel=0.2,seed=2",
    "groupby:rows=6000000,keys=1500000,zipf=0,seed=3",
    "groupby:rows=6000000,keys=1500000,zipf=0.5,seed=3",
    "groupby:rows=6000000,keys=1500000,zipf=1.0,seed=3",
    "groupby:rows=6000000,keys=1500000,zipf=1.25,seed=3",
    "star:rows=60000000,seed=4",
]


@pytest.mark.parametrize("spec", FULL)
def test_full_size_vs_oracle(spec):
    w = workload(spec)
    data = generate_workload_host(w)
    expect = result_lines(run_plan(w.plan, data))
    # the device generator produces the same columns; run from them (no host upload)
    e = Engine(0)
    e.load_workload(w, on_device=True)
    for flavor in ["", "cuda(load=tma)", "cuda(build=staged,aggr=cache)", "cuda(build=direct)", "cuda(aggr=part)",
                   "cuda(aggr=part,threads=512,parts=256)", "cuda(frows=1)",
                   "cuda(lowcard=regs)", "cuda(lowcard=regs,load=tma,rows=8)", "cuda(aggr=direct)",
                   "cuda(aggr=dcache)", "cuda(aggr=dcache,cache=256,threads=512,rows=2)"]:
        q = e.query(w.plan, flavor)
        q.run()
        assert q.result_lines() == expect, flavor
        q.close()


def test_device_generator_matches_host():
    w = workload("star:rows=100003,dates=2556,custs=3001,supps=200,parts=14011,seed=9")
    data = generate_workload_host(w)
    e = Engine(0)
    e.load_workload(w, on_device=True)
    for c in w.columns:
        assert np.array_equal(e.download(c.table, c.name), data[c.table][c.name]), c.name
    wz = workload("groupby:rows=200001,keys=5000,zipf=1.1,seed=9")
    dz = generate_workload_host(wz)
    ez = Engine(0)
    ez.load_workload(wz, on_device=True)
    for c in wz.columns:
        assert np.array_equal(ez.download(c.table, c.name), dz[c.table][c.name]), c.name


EDGE_SPECS = [
    "sel_aggr:rows=0,seed=5",
    "sel_aggr:rows=1,seed=5",
    "sel_aggr:rows=1023,seed=5",
    "sel_aggr:rows=4097,sel=0,seed=5",
    "join_aggr:build=0,probe=1000,seed=5",
    "join_aggr:build=1000,probe=0,seed=5",
    "join_aggr:build=1,probe=77,sel=1,seed=5",
    "groupby:rows=0,keys=10,seed=5",
    "groupby:rows=33,keys=1,seed=5",
    "groupby:rows=100000,keys=100000,zipf=1.25,seed=5",
    "star:rows=0,seed=5",
    "star:rows=999,dates=7,custs=1,supps=1,parts=1,seed=5",
]


@pytest.mark.parametrize("spec", EDGE_SPECS)
@pytest.mark.parametrize("flavor", ["", "cuda(rows=2,threads=32,aggr=global)", "cuda(load=tma,build=staged)",
                                    "cuda(build=direct,rows=1)", "cuda(aggr=part,rows=1,threads=64)"])
def test_edge_cases_vs_oracle(spec, flavor):
    """Empty and ragged inputs, no matches, single keys (the reference itself asserts on
    empty base tables, codegen.cpp:445, so the oracle is the only checker there)."""
    w = workload(spec)
    data = generate_workload_host(w)
    expect = result_lines(run_plan(w.plan, data))
    assert run_gpu(w, w.plan, flavor, data=data) == expect


def test_rerun_and_reset_are_idempotent():
    w = workload("groupby:rows=300000,keys=20000,zipf=1.0,seed=6")
    data = generate_workload_host(w)
    expect = result_lines(run_plan(w.plan, data))
    e = Engine(0)
    e.load_workload(w, data=data)
    for flavor in ["cuda(aggr=cache)", "cuda(aggr=part)"]:
        q = e.query(w.plan, flavor)
        for _ in range(3):
            q.run()
            assert q.result_lines() == expect, flavor
            q.reset()
        q.close()


def test_capacity_error_is_reported_not_faulted():
    """A join whose declared key domain is violated still cannot corrupt memory: keys outside
    the build domain never match, and the engine reports errors through status codes."""
    e = Engine(0)
    e.create_table("b", 4)
    e.add_column("b", "k", "i32", 1, 4)
    e.upload("b", "k", np.array([1, 2, 3, 4], dtype=np.int32))
    e.create_table("p", 6)
    e.add_column("p", "k", "i32", 0, 10)
    e.upload("p", "k", np.array([0, 1, 4, 5, 10, 2], dtype=np.int32))
    q = e.query("(aggr global () ((fun count)) (join join01 ((col p.k)) () (scan p (k)) ((col b.k)) () (scan b (k))))")
    q.run()
    assert q.result_lines() == ["3"]
