"""The chooser's host side without a GPU: plan-derived features (plan text alone is enough),
the per-kind knob grids and the reference-schema run log."""
import sqlite3

import numpy as np
import pytest

from vldb_voila_b200 import Engine, VoilaError, workload
from vldb_voila_b200 import chooser as ch


def test_grids_cover_each_kind_and_compile_offline():
    assert set(ch.GRIDS) == {"scan", "hash", "join", "star"}
    for k, g in ch.GRIDS.items():
        assert g[0] == ch.DEFAULT and len(set(g)) == len(g) >= 30, k
        assert set(g) <= set(ch.CANDIDATES)
    kinds = {"sel_aggr:rows=1000": "scan", "groupby:rows=1000,keys=100000": "hash",
             "join_aggr:build=100,probe=1000": "join", "star:rows=1000": "star"}
    for spec, kind in kinds.items():
        assert ch.kind_of(ch.describe_spec(spec)) == kind
        w = workload(spec)
        e = Engine(offline=True)
        e.load_workload(w)
        ok = 0
        for fl in ch.GRIDS[kind][:6] + ch.GRIDS[kind][-3:]:
            try:
                e.query(w.plan, fl)
                ok += 1
            except VoilaError as ex:
                assert ex.code == 6  # over the shared-memory limit: the autotuner skips it
        assert ok >= 6


def test_plan_text_alone_is_featurized():
    """A plan that arrives as text (no workload spec) gets the same features as the spec path
    when given the same statistics."""
    spec = "star:rows=5000,seed=3"
    w = workload(spec)
    e = Engine(offline=True)
    e.load_workload(w)
    desc = e.describe(w.plan)
    f = ch.plan_features(desc, 1 / 875.0, 0.0)
    assert f.shape == (len(ch.FEATURE_NAMES),)
    assert np.allclose(f, ch.features(spec))
    p = ch.fact_pipeline(desc)
    assert p["probes"] == 4 and p["sink"] == "aggr_dense" and p["rows"] == 5000
    # a plan no spec names: a hand-written join over the same tables
    plan = ("(aggr hash ((col customer.c_region)) ((fun sum (col lineorder.lo_revenue)))"
            " (join join01 ((col lineorder.lo_custkey)) () (scan lineorder (lo_custkey lo_revenue))"
            " ((col customer.c_custkey)) ((col customer.c_region)) (scan customer (c_custkey c_region))))")
    d2 = e.describe(plan)
    assert ch.kind_of(d2) == "join"
    f2 = ch.plan_features(d2)
    assert f2[ch.FEATURE_NAMES.index("probes")] == 1 and f2[ch.FEATURE_NAMES.index("kind_join")] == 1


def test_run_log_uses_the_reference_runs_schema(tmp_path):
    db = str(tmp_path / "voila.db")
    log = ch.RunLog(sqlite_path=db)
    log.record("full", "star:rows=5", "cuda(rows=8)", "OK", 0, 0.25, 5, 12.0)
    log.close()
    con = sqlite3.connect(db)
    cols = [r[1] for r in con.execute("PRAGMA table_info(runs)")]
    # the columns of compiler.cpp:104-110, in order
    assert cols == ["id", "t", "mode", "query", "result", "rep", "time_ms", "tuples", "cycles", "instructions",
                    "L1misses", "LLCmisses", "branchmisses", "taskclock", "threads", "cgen_ms", "ccomp_ms",
                    "default_blend", "key_check_blend", "aggregates_blend", "backend", "scale_factor",
                    "pipeline_flavor", "full_blend"]
    row = con.execute("SELECT mode, query, result, time_ms, backend, full_blend FROM runs").fetchone()
    assert row == ("full", "star:rows=5", "OK", 0.25, "cuda", "cuda(rows=8)")
