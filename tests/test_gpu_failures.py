"""Failure paths, made on the host and never by faulting the GPU: a batch work item whose
dependency never completes (its bounded wait runs out, the kernel returns and the batch
reports VC_ERR_TIMEOUT), and a group table that a flavor sized too small (bounded probe
sequences run out, the run reports VC_ERR_CAPACITY).  After each, the same device context
runs the queries again and gets the oracle's results."""
import numpy as np
import pytest

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, VoilaError, generate_workload_host, workload
from vldb_voila_b200.engine import Batch

pytestmark = pytest.mark.gpu

SPECS = ["join_aggr:build=20000,probe=100000,sel=0.3,seed=31", "groupby:rows=100000,keys=20000,zipf=0.5,seed=32",
         "sel_aggr:rows=100000,seed=33"]


def _queries(specs):
    engines, queries, expect = [], [], []
    for s in specs:
        w = workload(s)
        data = generate_workload_host(w)
        e = Engine(0)
        e.load_workload(w, data=data)
        engines.append(e)
        queries.append(e.query(w.plan))
        expect.append(result_lines(run_plan(w.plan, data)))
    return engines, queries, expect


def test_batch_dependency_wait_runs_out_and_the_kernel_returns():
    engines, queries, expect = _queries(SPECS)
    b = Batch(queries, tiles_per_item=2)
    b.run()
    b.wait()
    items = b.items()
    F = {k: i for i, k in enumerate(Batch.ITEM_FIELDS)}
    # a probe item of the join query: it waits for the join build's done-counter
    waiting = [i for i, r in enumerate(items) if r[F["shape"]] >= 0 and r[F["dep"]] >= 2]
    assert waiting
    b.set_wait_limit(1_000_000)  # 1 ms
    b.hold_item(waiting[0])
    b.run()
    with pytest.raises(VoilaError) as e:
        b.wait()
    assert e.value.code == 4  # VC_ERR_TIMEOUT
    # the kernel returned (the wait above ended) and the context is usable: release the
    # item and the batch gives every query its oracle result again
    b.hold_item(waiting[0], False)
    b.run()
    b.wait()
    for q, ex in zip(queries, expect):
        assert q.result_lines() == ex


@pytest.mark.parametrize("aggr", ["global", "cache"])
def test_undersized_group_table_reports_capacity(aggr):
    spec = "groupby:rows=60000,keys=20000,zipf=0.0,seed=34"
    w = workload(spec)
    data = generate_workload_host(w)
    e = Engine(0)
    e.load_workload(w, data=data)
    # ~17,000 distinct keys into 1,024 slots: probe sequences run out
    q = e.query(w.plan, f"cuda(aggr={aggr},gcap=1024)")
    q.run()
    with pytest.raises(VoilaError) as err:
        q.result_lines()
    assert err.value.code == 3  # VC_ERR_CAPACITY
    ok = e.query(w.plan, f"cuda(aggr={aggr})")
    ok.run()
    assert ok.result_lines() == result_lines(run_plan(w.plan, data))
    # the undersized query itself still runs cleanly once its input fits its table
    assert q.info()["flavor"].find("gcap=1024") >= 0
