"""Aggregations below the plan root kept on the device: the sub-aggregation's rows go to an
intermediate table (aggr_ht<N>.key_<i>, aggr_ht<N>.aggr_<j>, named as the reference's
translator names them) that a later pipeline of the same query scans, with the row count
read on the device.  The golden cases (agg_of_agg, having_*) pin this against the reference;
here more shapes are checked against the oracle, among them a sub-aggregation used as a
join's build side and as its probe side (the reference's code generator fails on the
former, so the oracle is the only check for it)."""
import pytest

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, generate_workload_host, workload

pytestmark = pytest.mark.gpu

SPEC = "groupby:rows=300000,keys=20000,zipf=0.9,seed=81"
PLANS = {
    # q18 shape: orders (here: keys) whose summed quantity passes a threshold, joined back
    "semi_join_build": (
        "(aggr global () ((fun sum (col lineitem.l_extendedprice)) (fun count))"
        " (join join01 ((col lineitem.l_orderkey)) () (scan lineitem (l_orderkey l_extendedprice))"
        " ((col aggr_ht2.key_0)) ()"
        " (select (fun > (col aggr_ht2.aggr_0) (const 150))"
        " (aggr hash ((col lineitem.l_orderkey)) ((fun sum (col lineitem.l_quantity))) (scan lineitem (l_orderkey l_quantity))))))"),
    # the aggregated rows probe a table built from the base rows (the join takes the
    # translator's id 0 before its build side, so the aggregation below it is aggr_ht2)
    "agg_probes": (
        "(aggr hash ((col aggr_ht2.aggr_1)) ((fun sum (col lineitem.l_quantity)) (fun count))"
        " (join joinN ((col aggr_ht2.key_0)) ()"
        "  (aggr hash ((col lineitem.l_orderkey)) ((fun sum (col lineitem.l_extendedprice)) (fun count))"
        "   (scan lineitem (l_orderkey l_extendedprice)))"
        "  ((col lineitem.l_orderkey)) ((col lineitem.l_quantity)) (scan lineitem (l_orderkey l_quantity))))"),
    # three levels
    "three_levels": (
        "(aggr global () ((fun sum (col aggr_ht3.aggr_0)) (fun count))"
        " (aggr hash ((col aggr_ht1.aggr_1)) ((fun sum (col aggr_ht1.aggr_0)))"
        "  (aggr hash ((col lineitem.l_orderkey)) ((fun sum (col lineitem.l_quantity)) (fun count))"
        "   (scan lineitem (l_orderkey l_quantity)))))"),
    # a projection over the aggregated columns, then a grouped aggregate
    "project_over_agg": (
        "(aggr hash ((col big)) ((fun sum (col aggr_ht1.aggr_0)) (fun count))"
        " (project ((assign big (fun - (col aggr_ht1.aggr_1) (const 20))) (col aggr_ht1.aggr_0))"
        "  (aggr hash ((col lineitem.l_orderkey)) ((fun sum (col lineitem.l_quantity)) (fun count))"
        "   (scan lineitem (l_orderkey l_quantity)))))"),
}
FLAVORS = ["", "cuda(aggr=cache,cache=128)", "cuda(load=tma,stages=3,rows=8)", "cuda(rows=1,threads=64,graph=0)"]


@pytest.fixture(scope="module")
def db():
    w = workload(SPEC)
    data = generate_workload_host(w)
    e = Engine(0)
    e.load_workload(w, data=data)
    return data, e


@pytest.mark.parametrize("flavor", FLAVORS)
@pytest.mark.parametrize("name", sorted(PLANS))
def test_sub_aggregation_matches_oracle(db, name, flavor):
    data, e = db
    plan = PLANS[name]
    expect = result_lines(run_plan(plan, data))
    assert expect
    q = e.query(plan, flavor)
    for _ in range(2):
        q.run()
        assert q.result_lines() == expect
    q.close()
