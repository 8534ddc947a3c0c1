"""The batched persistent kernel: every query of a mixed batch gets exactly the result it
gets on its own (and the oracle's), over repeated graph replays."""
import numpy as np
import pytest

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, generate_workload_host, workload
from vldb_voila_b200.engine import Batch, batch_specs

pytestmark = pytest.mark.gpu


def _setup(specs, flavor_of=lambda s: ""):
    engines, queries, expect = [], [], []
    for s in specs:
        w = workload(s)
        data = generate_workload_host(w)
        e = Engine(0)
        e.load_workload(w, data=data)
        engines.append(e)
        queries.append(e.query(w.plan, flavor_of(s)))
        expect.append(result_lines(run_plan(w.plan, data)))
    return engines, queries, expect


def test_mixed_batch_matches_oracle_and_is_repeatable():
    specs = batch_specs(24, seed=3, min_rows=1_000, max_rows=400_000)
    specs += ["star:rows=50000,custs=3000,supps=200,parts=14000,seed=9", "groupby:rows=0,keys=10,seed=1",
              "sel_aggr:rows=1,seed=2", "join_aggr:build=0,probe=100,seed=3"]
    engines, queries, expect = _setup(specs)
    for s, q, e in zip(specs, queries, expect):
        q.run()
        assert q.result_lines() == e, s
    b = Batch(queries, tiles_per_item=2)
    assert b.info()["work_items"] >= len(specs)
    for _ in range(3):
        b.run()
        b.wait()
        for s, q, e in zip(specs, queries, expect):
            assert q.result_lines() == e, s
    lat = b.latencies_us()
    assert all(x >= 0 for x in lat)
    # the same queries still run on their own afterwards
    for s, q, e in zip(specs, queries, expect):
        q.run()
        assert q.result_lines() == e, s


def test_split_batch_runs_large_queries_on_their_own():
    """vc_batch_new_split: queries with a pipeline of at least solo_rows rows run as their own
    launches after the persistent kernel; every query still gets the oracle's rows, over
    repeated runs, and every query has a latency."""
    specs = batch_specs(16, seed=6, min_rows=1_000, max_rows=300_000)
    specs += ["groupby:rows=0,keys=10,seed=1"]
    engines, queries, expect = _setup(specs)
    rows = [workload(s).fact_rows for s in specs]
    cut = sorted(rows)[len(rows) // 2]
    b = Batch(queries, tiles_per_item=2, solo_rows=cut)
    info = b.info()
    assert info["solo"] >= 1 and info["batched"] >= 1 and info["solo"] + info["batched"] == len(specs)
    for _ in range(2):
        b.run()
        b.wait()
        for s, q, e in zip(specs, queries, expect):
            assert q.result_lines() == e, s
    lat = b.latencies_us()
    assert len(lat) == len(specs) and all(x >= 0 for x in lat)
    # every query with a row on its own: only the empty one stays in the persistent kernel
    alone = Batch(queries, solo_rows=1)
    assert alone.info()["batched"] == sum(1 for r in rows if r == 0)
    alone.run()
    alone.wait()
    for s, q, e in zip(specs, queries, expect):
        assert q.result_lines() == e, s


def test_batch_with_per_query_flavors():
    specs = batch_specs(12, seed=4, min_rows=10_000, max_rows=200_000)
    choice = ["cuda(lowcard=private)", "cuda(aggr=cache,cache=128)", "cuda(prefetch=0,rows=2)", ""]
    engines, queries, expect = _setup(specs)
    b = Batch(queries, flavors=[choice[i % 4] for i in range(len(specs))], threads=128, tiles_per_item=4)
    b.run()
    b.wait()
    for q, e in zip(queries, expect):
        assert q.result_lines() == e


def test_batch_mixing_smem_and_probe_heavy_shapes():
    """Dense shared-memory group-bys, the shared-memory group cache and the plain hash
    group-by in one persistent kernel.  Warps leave the hash probe loops at different times;
    this mix once made the warps of a CTA drift onto different work items at a block
    barrier, so every run of it is checked against the oracle."""
    specs = batch_specs(12, seed=4, min_rows=10_000, max_rows=200_000)
    cache, lean = "cuda(aggr=cache,cache=128)", "cuda(prefetch=0,rows=2)"
    choice = ["", cache, lean, ""]
    engines, queries, expect = _setup(specs)
    b = Batch(queries, flavors=[choice[i % 4] for i in range(len(specs))], threads=128, tiles_per_item=4)
    for _ in range(4):
        b.run()
        b.wait()
        for s, q, e in zip(specs, queries, expect):
            assert q.result_lines() == e, s


def test_batch_with_a_join_whose_build_side_is_a_join():
    """The customer table's build probes the date table: inside the persistent kernel it must
    wait for the date build, or it silently misses rows."""
    from helpers import NESTED_BUILD_PLAN
    spec = "star:rows=200000,custs=30000,supps=200,parts=14000,seed=11"
    w = workload(spec)
    data = generate_workload_host(w)
    e = Engine(0)
    e.load_workload(w, data=data)
    expect = result_lines(run_plan(NESTED_BUILD_PLAN, data))
    assert expect and expect[0] != "0|0"
    q = e.query(NESTED_BUILD_PLAN)
    q.run()
    assert q.result_lines() == expect
    others, oq, oexp = _setup(batch_specs(6, seed=8, min_rows=10_000, max_rows=200_000))
    b = Batch([q] + oq, tiles_per_item=2)
    for _ in range(3):
        b.run()
        b.wait()
        assert q.result_lines() == expect
        for x, ex in zip(oq, oexp):
            assert x.result_lines() == ex
