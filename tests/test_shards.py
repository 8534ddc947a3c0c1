"""The multi-GPU exchange step on CPU: world-size-2 gloo ranks each aggregate a row range of
the fact table (build tables replicated) and merge partials; the merged result equals the
oracle over the whole table."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

SPECS = ["sel_aggr:rows=40000,seed=5", "groupby:rows=50000,keys=7000,zipf=1.1,seed=6",
         "join_aggr:build=4000,probe=30000,sel=0.4,seed=7", "star:rows=30000,custs=500,supps=50,parts=900,seed=8"]
# an emit plan (no aggregation at the root): the ranks' rows are concatenated, never summed
EMIT_PLAN = ("(select (fun < (col lineitem.l_val) (const 200000)) "
             "(join join01 ((col lineitem.l_orderkey)) () (scan lineitem (l_orderkey l_val)) "
             "((col orders.o_orderkey)) ((col orders.o_attr)) (scan orders (o_orderkey o_attr))))")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, spec, q, plan=None):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.voila_oracle import parse_sexpr, run_plan
        from vldb_voila_b200 import generate_workload_host, workload
        from vldb_voila_b200.shards import gather_result, merge_partials, shard_rows
        from vldb_voila_b200.shards import plan_group_keys
        w = workload(spec)
        if plan is not None:
            w.plan = plan
        data = generate_workload_host(w)
        b, e = shard_rows(w.fact_rows, rank, world)
        shard = {t: dict(cols) for t, cols in data.items()}
        shard[w.fact_table] = {c: v[b:e] for c, v in data[w.fact_table].items()}
        node = parse_sexpr(w.plan)
        nkeys = plan_group_keys(w.plan)
        assert nkeys == (len(node[2]) if node[0] == "aggr" and node[1] == "hash" else
                         (0 if node[0] == "aggr" else -1))
        part = np.array(run_plan(w.plan, shard), dtype=np.int64)
        ncols = len(run_plan(w.plan, data)[0])
        merged = merge_partials(part.reshape(-1, ncols), nkeys, ncols)
        full = gather_result(merged, ncols)
        if rank == 0:
            q.put(sorted(map(tuple, full.tolist())) == sorted(run_plan(w.plan, data)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("spec,plan", [(s, None) for s in SPECS] +
                         [("join_aggr:build=3000,probe=20000,seed=9", EMIT_PLAN)])
def test_two_ranks_merge_to_the_whole_result(spec, plan):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, spec, q, plan)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        assert p.exitcode == 0
    assert q.get(timeout=10) is True


def test_plan_group_keys_classifies_plan_roots():
    from vldb_voila_b200.shards import EMIT, merge_rows, plan_group_keys
    assert plan_group_keys("(aggr hash ((col a.x) (col a.y)) ((fun count)) (scan a (x y)))") == 2
    assert plan_group_keys("(aggr global () ((fun count)) (scan a (x)))") == 0
    assert plan_group_keys(EMIT_PLAN) == EMIT
    with pytest.raises(ValueError):
        plan_group_keys("scan")
    with pytest.raises(ValueError):
        merge_rows(np.zeros((2, 2), dtype=np.int64), EMIT, 0, 2)
