"""Columns that stay in pinned host memory (vc_column_attach_host): the kernels read them in
place over PCIe and every result equals the oracle's, for eager scans, lazily gathered probe
columns and a flavor that asks for bulk copies (which host-resident columns do not use)."""
import numpy as np
import pytest
import torch

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import Engine, VoilaError, generate_workload_host, workload

pytestmark = pytest.mark.gpu

SPECS = ["star:rows=300000,custs=3000,supps=200,parts=14000,seed=71", "join_aggr:build=20000,probe=200000,seed=72",
         "sel_aggr:rows=200000,seed=73", "groupby:rows=200000,keys=30000,zipf=1.0,seed=74"]


def _host_engine(w, data):
    e = Engine(0)
    keep = []
    for t, rows in w.tables.items():
        e.create_table(t, rows)
    for c in w.columns:
        e.add_column(c.table, c.name, c.type, c.lo, c.hi)
        a = np.ascontiguousarray(data[c.table][c.name])
        pinned = torch.from_numpy(a.view(np.uint8)).pin_memory()
        keep.append(pinned)
        e.attach_host(c.table, c.name, pinned.data_ptr())
    return e, keep


@pytest.mark.parametrize("flavor", ["", "cuda(load=tma,stages=3)", "cuda(rows=8,compact=-1)"])
@pytest.mark.parametrize("spec", SPECS)
def test_host_resident_columns_match_oracle(spec, flavor):
    w = workload(spec)
    data = generate_workload_host(w)
    e, keep = _host_engine(w, data)
    q = e.query(w.plan, flavor)
    expect = result_lines(run_plan(w.plan, data))
    for _ in range(2):
        q.run()
        assert q.result_lines() == expect
    assert "bulk_load" not in q.source()  # bulk copies never read host memory
    q.close()
    e.close()


def test_attach_host_rejects_pageable_memory():
    e = Engine(0)
    e.create_table("t", 16)
    e.add_column("t", "x", "i64", 0, 10)
    a = np.zeros(16, dtype=np.int64)
    with pytest.raises(VoilaError) as ex:
        e.attach_host("t", "x", a.ctypes.data)
    assert ex.value.code == 1
