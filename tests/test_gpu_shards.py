"""The sharded path through the CUDA flavor: each rank's row range of the fact table runs as
its own query (here the ranks run one after another on one GPU; nothing waits across them),
and the exchange step's merge of their partial rows equals the oracle over the whole table."""
import numpy as np
import pytest

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, generate_workload_host, workload
from vldb_voila_b200.shards import EMIT, load_shard, merge_rows, plan_group_keys

pytestmark = pytest.mark.gpu

SPECS = ["sel_aggr:rows=400000,seed=5", "groupby:rows=500000,keys=70000,zipf=1.1,seed=6",
         "join_aggr:build=40000,probe=300000,sel=0.4,seed=7",
         "star:rows=300000,custs=5000,supps=500,parts=9000,seed=8"]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("spec", SPECS)
def test_cuda_shards_merge_to_the_whole_result(spec, world):
    w = workload(spec)
    data = generate_workload_host(w)
    nkeys = plan_group_keys(w.plan)
    assert nkeys != EMIT
    parts = []
    for rank in range(world):
        e = Engine(0)
        load_shard(e, w, data, rank, world)
        q = e.query(w.plan)
        q.run()
        parts.append(q.result())
        q.close()
        e.close()
    allrows = np.concatenate(parts, axis=0)
    merged = np.concatenate([merge_rows(allrows, nkeys, r, world) for r in range(world)], axis=0)
    got = sorted("|".join(str(v) for v in row) for row in merged.tolist())
    assert got == result_lines(run_plan(w.plan, data))
