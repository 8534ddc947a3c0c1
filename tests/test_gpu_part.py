"""Partitioned hash aggregation (flavor aggr=part) against the oracle: partitions split over
several work items and merged by the last one, a single hot key, empty input, and records
of two words."""
import pytest

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, generate_workload_host, workload

pytestmark = pytest.mark.gpu


def check(spec, flavor, runs=2):
    w = workload(spec)
    data = generate_workload_host(w)
    expect = result_lines(run_plan(w.plan, data))
    e = Engine(0)
    e.load_workload(w, data=data)
    q = e.query(w.plan, flavor)
    for _ in range(runs):
        q.run()
        assert q.result_lines() == expect, (spec, flavor)
    q.close()
    e.close()


@pytest.mark.parametrize("spec", [
    # 16 partitions of ~19K records each: every partition is split over two items (R = 16384)
    "groupby:rows=300000,keys=20000,zipf=0,seed=11",
    "groupby:rows=300000,keys=20000,zipf=1.25,seed=11",
    # one key: all records in one partition, 13 items merged by the last
    "groupby:rows=200000,keys=1,seed=12",
    "groupby:rows=0,keys=10,seed=13",
    "groupby:rows=5,keys=1000000,seed=13",
])
@pytest.mark.parametrize("flavor", ["cuda(aggr=part,parts=16)", "cuda(aggr=part,parts=2048,threads=512,rows=8)",
                                    "cuda(aggr=part,threads=64,rows=2)"])
def test_partitioned_aggregation_vs_oracle(spec, flavor):
    check(spec, flavor)


def test_two_word_records():
    # sums of values spanning about 2^52 beside a 16-bit key: records of two words
    check("bigsum:rows=40000,seed=95", "cuda(aggr=part)")


def test_partitioned_sub_aggregation():
    from helpers import manifest
    m = manifest()["agg_of_agg"]
    w = workload(m["spec"])
    data = generate_workload_host(w)
    expect = result_lines(run_plan(m["plan"], data))
    e = Engine(0)
    e.load_workload(w, data=data)
    q = e.query(m["plan"], "cuda(aggr=part)")
    q.run()
    assert q.result_lines() == expect


def test_batched_partitioned_query_matches_standalone():
    """A batch takes a query prepared with aggr=part through the global group table; the
    query still runs standalone with its partitioned kernels afterwards."""
    from vldb_voila_b200.engine import Batch
    spec = "groupby:rows=300000,keys=20000,zipf=1.0,seed=14"
    w = workload(spec)
    data = generate_workload_host(w)
    expect = result_lines(run_plan(w.plan, data))
    e = Engine(0)
    e.load_workload(w, data=data)
    q = e.query(w.plan, "cuda(aggr=part)")
    b = Batch([q])
    for _ in range(2):
        b.run()
        b.wait()
        assert q.result_lines() == expect
    q.run()
    assert q.result_lines() == expect
