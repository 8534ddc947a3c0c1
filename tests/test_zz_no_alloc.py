"""The allocation-free join + aggregate entry point (vc_join_aggr_noalloc), for callers that
cannot allocate device memory, checked through the C ABI against the regular query path
(a join_aggr query) on two calls in a row.  Collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fn():
    from vldb_voila_b200.engine import lib
    f = lib().vc_join_aggr_noalloc
    P = ctypes.c_void_p
    f.restype = ctypes.c_int
    f.argtypes = [P, P, ctypes.c_int64, ctypes.c_int32, P, P, ctypes.c_int64, P, P]
    return f


def _reference(e, plan):
    q = e.query(plan)
    q.run()
    rows = q.result()
    q.close()
    return (int(rows[0, 0]), int(rows[0, 1])) if len(rows) else (0, 0)


@pytest.mark.parametrize("spec", ["join_aggr:build=1500000,probe=6000000,sel=0.2,seed=2",
                                  "join_aggr:build=20000,probe=100000,sel=0.7,seed=21"])
def test_noalloc_matches_the_query_path_twice(spec):
    import torch
    from vldb_voila_b200 import Engine, workload
    from vldb_voila_b200.engine import check
    w = workload(spec)
    e = Engine(0)
    e.load_workload(w, on_device=True)
    torch.cuda.synchronize()
    expect = _reference(e, w.plan)
    thr = int(w.plan.split("(fun < (col orders.o_attr) (const ")[1].split(")")[0])
    ptr = lambda t, c: ctypes.c_void_p(e.device_ptr(t, c))
    out = torch.full((3,), -1, dtype=torch.int64, device="cuda")
    f = _fn()
    for _ in range(2):
        out.fill_(-1)
        torch.cuda.synchronize()
        check(f(ptr("orders", "o_orderkey"), ptr("orders", "o_attr"), w.tables["orders"], thr,
                ptr("lineitem", "l_orderkey"), ptr("lineitem", "l_val"), w.tables["lineitem"],
                ctypes.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        got = out.cpu().tolist()
        assert got[2] == 0
        assert (got[0], got[1]) == expect


def test_noalloc_rejects_oversized_builds():
    from vldb_voila_b200.engine import VoilaError, check
    f = _fn()
    with pytest.raises(VoilaError) as ex:
        check(f(ctypes.c_void_p(16), ctypes.c_void_p(16), 2_097_153, 0, None, None, 0, ctypes.c_void_p(16), None))
    assert ex.value.code == 1 and "2097152" in str(ex.value)


def test_noalloc_negative_and_duplicate_build_keys():
    """Negative keys and build keys that repeat (Join01 keeps one match per probe row), on
    both paths; out[2] (the error bits) must be read on every VC_OK return."""
    import torch
    from oracle.voila_oracle import run_plan
    from vldb_voila_b200 import Engine
    from vldb_voila_b200.engine import check
    rng = np.random.default_rng(5)
    nb, npr, thr = 5000, 40000, 40
    cols = {"orders": {"o_orderkey": rng.integers(-3000, 3000, nb).astype(np.int32),
                       "o_attr": rng.integers(0, 100, nb).astype(np.int32)},
            "lineitem": {"l_orderkey": rng.integers(-3500, 3500, npr).astype(np.int32),
                         "l_val": rng.integers(-1000, 1000000, npr).astype(np.int64)}}
    assert len(np.unique(cols["orders"]["o_orderkey"])) < nb  # duplicates present
    e = Engine(0)
    e.create_table("orders", nb)
    e.add_column("orders", "o_orderkey", "i32", -3000, 2999)
    e.add_column("orders", "o_attr", "i32", 0, 99)
    e.create_table("lineitem", npr)
    e.add_column("lineitem", "l_orderkey", "i32", -3500, 3499)
    e.add_column("lineitem", "l_val", "i64", -1000, 999999)
    for t, cs in cols.items():
        for c, a in cs.items():
            e.upload(t, c, a)
    plan = ("(aggr global () ((fun sum (col lineitem.l_val)) (fun count))"
            " (join join01 ((col lineitem.l_orderkey)) () (scan lineitem (l_orderkey l_val))"
            " ((col orders.o_orderkey)) ()"
            f" (select (fun < (col orders.o_attr) (const {thr})) (scan orders (o_orderkey o_attr)))))")
    expect = _reference(e, plan)
    assert [list(expect)] == [list(r) for r in run_plan(plan, cols)]
    ptr = lambda t, c: ctypes.c_void_p(e.device_ptr(t, c))
    out = torch.full((3,), -1, dtype=torch.int64, device="cuda")
    f = _fn()
    for _ in range(2):
        out.fill_(-1)
        torch.cuda.synchronize()
        check(f(ptr("orders", "o_orderkey"), ptr("orders", "o_attr"), nb, thr, ptr("lineitem", "l_orderkey"),
                ptr("lineitem", "l_val"), npr, ctypes.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        got = out.cpu().tolist()
        assert got[2] == 0
        assert (got[0], got[1]) == expect
