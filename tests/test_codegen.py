"""Plan lowering, CUDA code generation and NVRTC compilation for sm_100a, on an offline
(compile-only) engine: runs on a build host without a GPU."""
import pytest

from vldb_voila_b200 import Engine, VoilaError, workload

SPECS = ["sel_aggr:rows=1000", "join_aggr:build=100,probe=1000", "groupby:rows=1000,keys=100000,zipf=1.0",
         "groupby:rows=1000,keys=50", "star:rows=1000"]
FLAVORS = ["", "cuda(load=tma,stages=2)", "cuda(lowcard=private,prefetch=0)", "cuda(aggr=cache,build=staged)",
           "cuda(compact=0,rows=8,threads=128)", "cuda(hash=voila,compact=-1)", "cuda(build=direct,prefetch=0)",
           "cuda(lowcard=redux,aggr=cache,cache=64)", "cuda(lowcard=atomic,sinksmem=4096)"]


def offline(spec):
    w = workload(spec)
    e = Engine(offline=True)
    e.load_workload(w)
    return w, e


@pytest.mark.parametrize("spec", SPECS)
@pytest.mark.parametrize("flavor", FLAVORS)
def test_workload_plans_compile_for_sm100a(spec, flavor):
    w, e = offline(spec)
    q = e.query(w.plan, flavor)
    info = q.info()
    src = q.source()
    assert any(k["dominant"] for k in info["kernels"])
    assert "vc_p0_main" in src
    if w.template == "join_aggr":
        # small key spaces get a dense (direct-address) table unless a hash build is forced
        hashed = "build=staged" in flavor or "build=direct" in flavor
        assert ("join_probe_bucket" in src) == hashed
        assert ("vd::dense_test" in src) == (not hashed)
    if "load=tma" in flavor and w.template != "star":
        assert "vd::bulk_load" in src and "mbar_wait" in src


def test_pipeline_structure_follows_the_plan():
    w, e = offline("star:rows=1000")
    info = e.query(w.plan).info()
    sinks = [p["sink"] for p in info["pipelines"]]
    assert sinks == ["join_build"] * 4 + ["aggr_dense"]
    assert info["pipelines"][-1]["ops"] == 4


def test_shapes_share_generated_code_across_instances():
    w1, e1 = offline("groupby:rows=1000,keys=100000,zipf=1.0,seed=1")
    w2, e2 = offline("groupby:rows=5000,keys=200000,zipf=0.5,seed=2")
    assert e1.query(w1.plan).source() == e2.query(w2.plan).source()


@pytest.mark.parametrize("plan,code", [
    ("(scan lineitem (l_quantity)", 1),
    ("(scan nosuch (a))", 1),
    ("(select (fun < (col lineitem.l_nope) (const 1)) (scan lineitem (l_quantity)))", 1),
    ("(aggr global () ((fun min (col lineitem.l_quantity))) (scan lineitem (l_quantity)))", 6),
    ("(select (fun like (col lineitem.l_quantity) (const 1)) (scan lineitem (l_quantity)))", 6),
    # sum(price * price * price) over 1000 rows leaves int64: rejected, never wrapped
    ("(aggr global () ((fun sum (fun * (fun * (col lineitem.l_extendedprice) (col lineitem.l_extendedprice)) "
     "(col lineitem.l_extendedprice)))) (scan lineitem (l_extendedprice)))", 6),
])
def test_bad_or_unsupported_plans_fail_with_status(plan, code):
    w, e = offline("sel_aggr:rows=1000")
    with pytest.raises(VoilaError) as ex:
        e.query(plan)
    assert ex.value.code == code


def test_batch_module_compiles_and_dedups_shapes():
    from vldb_voila_b200.engine import Batch, batch_specs
    specs = batch_specs(9, seed=3, min_rows=1000, max_rows=400000) + ["star:rows=5000,seed=9"]
    engines, queries = [], []
    for s in specs:
        w, e = offline(s)
        engines.append(e)
        queries.append(e.query(w.plan))
    one = Batch(queries[:1])
    many = Batch(queries)
    # one persistent kernel; shapes shared: far less code than one copy per query
    assert many.info()["source_bytes"] < 4 * one.info()["source_bytes"] * 3
    assert many.info()["work_items"] >= len(specs)
    src = many.source()
    # a pipeline's item k strides its tiles by the pipeline's item count
    assert "t += nitems" in src
    # block barriers are the non-aligned form: warps may arrive diverged after probe loops
    assert "__syncthreads" not in src and "vd::block_sync()" in src


def test_batch_work_queue_only_waits_on_earlier_items():
    """CTAs of the persistent kernel claim items in queue order, so the queue is deadlock-free
    when every item's dependency is met by items before it; each query's clears also precede
    its first work item."""
    from collections import Counter

    from vldb_voila_b200.engine import Batch, batch_specs
    specs = batch_specs(12, seed=3, min_rows=1000, max_rows=400000)
    specs += ["star:rows=5000,seed=9", "join_aggr:build=1000,probe=5000,seed=4", "groupby:rows=0,keys=10,seed=1"]
    engines, queries = [], []
    for s in specs:
        w, e = offline(s)
        engines.append(e)
        queries.append(e.query(w.plan))
    b = Batch(queries, tiles_per_item=4)
    items = b.items()
    assert len(items) == b.info()["work_items"]
    F = {k: i for i, k in enumerate(Batch.ITEM_FIELDS)}
    produced = Counter()
    for row in items:
        if row[F["dep"]] >= 0:
            assert produced[row[F["dep"]]] >= row[F["dep_target"]]
        produced[row[F["done"]]] += 1
    clears = items[items[:, F["shape"]] == -1]
    work = items[items[:, F["shape"]] >= 0]
    assert len(clears) >= len(specs) and len(work) >= len(specs)
    # every first-phase work item waits for its own query's clears, which all precede it
    waits_on_clears = [r for r in work if r[F["dep"]] in set(clears[:, F["done"]])]
    assert waits_on_clears
    for r in waits_on_clears:
        assert produced[r[F["dep"]]] == r[F["dep_target"]]


@pytest.mark.parametrize("spec", SPECS)
def test_generated_kernels_use_non_aligned_barriers(spec):
    w, e = offline(spec)
    for flavor in ["", "cuda(load=tma,stages=2)", "cuda(compact=0)", "cuda(lowcard=private)"]:
        src = e.query(w.plan, flavor).source()
        assert "__syncthreads" not in src, flavor


def test_dense_join_tables_follow_the_key_space():
    # join_aggr's build keys span 1..1.5M: a bitmap of 2^21 bits beats a 2^22-slot hash table
    w, e = offline("join_aggr:build=1500000,probe=6000000,sel=0.2,seed=2")
    assert "vd::dense_test" in e.query(w.plan).source()
    assert "join_probe_bucket" in e.query(w.plan, "cuda(build=direct)").source()
    # star's dimension joins carry payloads: dense payload arrays
    w, e = offline("star:rows=1000")
    src = e.query(w.plan).source()
    assert "atomicCAS(&jdt" in src and "join_probe_bucket" not in src


@pytest.mark.parametrize("flavor", ["cuda(rows=3)", "cuda(threads=100)", "cuda(aggr=magic)", "gpu(x=1)", "cuda(nokey=1)"])
def test_bad_flavors_are_rejected(flavor):
    w, e = offline("sel_aggr:rows=1000")
    with pytest.raises(VoilaError) as ex:
        e.query(w.plan, flavor)
    assert ex.value.code == 1


def test_flavor_beyond_the_shared_memory_limit_is_rejected_at_creation():
    # an 8-row, 512-thread TMA tile ring with 4 stages needs more than 227 KiB per CTA
    w, e = offline("sel_aggr:rows=6000000")
    with pytest.raises(VoilaError) as ex:
        e.query(w.plan, "cuda(threads=512,rows=8,load=tma,stages=4)")
    assert ex.value.code == 6
    assert "shared memory" in str(ex.value)
