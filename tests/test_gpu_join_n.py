"""JoinN (multi-match) probes through the CUDA flavor against the oracle: every build row with
the probe row's key is a match and the rest of the pipeline runs once per match
(relalg_translator.cpp:1032-1042 without the Join01 exit).  Covers a grouped and a global
aggregate, an emitting plan (block-wide appends inside the match loop), a JoinN followed by a
Join01 probe, and skewed duplicate counts."""
import pytest

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, generate_workload_host, workload

pytestmark = pytest.mark.gpu

SPEC = "star:rows=40000,dates=100,custs=700,supps=10,parts=300,seed=61"
PLANS = {
    "grouped": "(aggr hash ((col customer.c_region)) ((fun sum (col lineorder.lo_revenue)) (fun count))"
               " (join joinN ((col customer.c_custkey)) () (scan customer (c_custkey c_region))"
               " ((col lineorder.lo_custkey)) ((col lineorder.lo_revenue)) (scan lineorder (lo_custkey lo_revenue))))",
    "global": "(aggr global () ((fun sum (col lineorder.lo_supplycost)) (fun count))"
              " (join joinN ((col part.p_partkey)) () (select (fun < (col part.p_category) (const 5))"
              " (scan part (p_partkey p_category)))"
              " ((col lineorder.lo_partkey)) ((col lineorder.lo_supplycost))"
              " (scan lineorder (lo_partkey lo_supplycost))))",
    "emit": "(select (fun < (col lineorder.lo_revenue) (const 3000000))"
            " (join joinN ((col customer.c_custkey)) () (scan customer (c_custkey c_region))"
            " ((col lineorder.lo_custkey)) ((col lineorder.lo_revenue)) (scan lineorder (lo_custkey lo_revenue))))",
    "chain": "(aggr hash ((col part.p_category)) ((fun sum (col lineorder.lo_revenue)) (fun count))"
             " (join join01 ((col lineorder.lo_partkey)) ()"
             "  (join joinN ((col customer.c_custkey)) () (scan customer (c_custkey c_mktsegment))"
             "   ((col lineorder.lo_custkey)) ((col lineorder.lo_partkey) (col lineorder.lo_revenue))"
             "   (scan lineorder (lo_custkey lo_partkey lo_revenue)))"
             "  ((col part.p_partkey)) ((col part.p_category)) (scan part (p_partkey p_category))))",
}
FLAVORS = ["", "cuda(build=staged)", "cuda(rows=1,threads=64,graph=0)", "cuda(load=tma,stages=3,aggr=cache,cache=64)",
           "cuda(hash=voila,rows=8)", "cuda(frows=1,compact=0)", "cuda(aggr=part,frows=2,compact=0)"]


@pytest.fixture(scope="module")
def star():
    w = workload(SPEC)
    data = generate_workload_host(w)
    e = Engine(0)
    e.load_workload(w, data=data)
    return w, data, e


@pytest.mark.parametrize("flavor", FLAVORS)
@pytest.mark.parametrize("name", sorted(PLANS))
def test_join_n_matches_oracle(star, name, flavor):
    w, data, e = star
    plan = PLANS[name]
    expect = result_lines(run_plan(plan, data))
    assert expect
    q = e.query(plan, flavor)
    for _ in range(2):
        q.run()
        assert q.result_lines() == expect
    q.close()


def test_join_n_with_skewed_duplicates():
    """Zipf-skewed build keys: a few keys repeat thousands of times, so the match loops of
    one warp have very different lengths."""
    spec = "groupby:rows=30000,keys=400,zipf=1.25,seed=62"
    w = workload(spec)
    data = generate_workload_host(w)
    e = Engine(0)
    e.load_workload(w, data=data)
    e.create_table("probe", 2000)
    e.add_column("probe", "pk", "i32", 1, 400)
    import numpy as np
    pk = (np.arange(2000) % 400 + 1).astype(np.int32)
    e.upload("probe", "pk", pk)
    data["probe"] = {"pk": pk}
    plan = ("(aggr global () ((fun sum (col lineitem.l_extendedprice)) (fun count))"
            " (join joinN ((col probe.pk)) () (scan probe (pk))"
            " ((col lineitem.l_orderkey)) ((col lineitem.l_extendedprice)) (scan lineitem (l_orderkey l_extendedprice))))")
    expect = result_lines(run_plan(plan, data))
    for fl in ["", "cuda(rows=8,threads=512)"]:
        q = e.query(plan, fl)
        q.run()
        assert q.result_lines() == expect
