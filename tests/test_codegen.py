"""Plan lowering, CUDA code generation and NVRTC compilation for sm_100a, on an offline
(compile-only) engine: runs on a build host without a GPU."""
import pytest

from helpers import NESTED_BUILD_PLAN
from vldb_voila_b200 import Engine, VoilaError, workload

SPECS = ["sel_aggr:rows=1000", "join_aggr:build=100,probe=1000", "groupby:rows=1000,keys=100000,zipf=1.0",
         "groupby:rows=1000,keys=50", "star:rows=1000"]
FLAVORS = ["", "cuda(load=tma,stages=2)", "cuda(lowcard=private,prefetch=0)", "cuda(aggr=cache,build=staged)",
           "cuda(compact=0,rows=8,threads=128)", "cuda(hash=voila,compact=-1)", "cuda(build=direct,prefetch=0)",
           "cuda(lowcard=redux,aggr=cache,cache=64)", "cuda(lowcard=atomic,sinksmem=4096)",
           "cuda(build=direct,probe=8)", "cuda(aggr=part)", "cuda(aggr=part,parts=16,threads=128,rows=8)",
           "cuda(aggr=part,load=tma,stages=2,compact=0)", "cuda(frows=1)", "cuda(frows=8,compact=0,aggr=part)",
           "cuda(lowcard=regs)", "cuda(lowcard=regs,load=tma,stages=2,rows=8,pgroups=4)",
           "cuda(aggr=direct)", "cuda(aggr=dcache,cache=256)", "cuda(lowcard=combine)",
           "cuda(lowcard=packed,load=tma,stages=2,pgroups=3)", "cuda(stream=noalloc)",
           "cuda(stream=noalloc,compact=0,rows=8)"]


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
    if "probe=" in flavor and w.template in ("join_aggr", "star"):
        assert "__ballot_sync(cmask" in src  # warp-cooperative probing
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
    # the accumulator words' bit fields follow the row-count bound: instances whose fields
    # have the same widths share one compiled shape, whatever their sizes, keys and skew
    w1, e1 = offline("groupby:rows=1000,keys=100000,zipf=1.0,seed=1")
    w2, e2 = offline("groupby:rows=1020,keys=200000,zipf=0.5,seed=2")
    assert e1.query(w1.plan).source() == e2.query(w2.plan).source()
    w3, e3 = offline("join_aggr:build=100,probe=1000,seed=1")
    w4, e4 = offline("join_aggr:build=300,probe=5000,seed=2")
    assert e3.query(w3.plan).source() == e4.query(w4.plan).source()


def test_hash_group_aggregates_share_accumulator_words():
    """sum(v1) (20-bit values), sum(v2) (6-bit) and count over 6M rows need 43, 29 and 23 bits:
    two 64-bit words, so each group update is two atomics instead of three."""
    w, e = offline("groupby:rows=6000000,keys=1500000,zipf=0.0,seed=3")
    src = e.query(w.plan, "cuda(aggr=global)").source()
    assert "uint64_t w[2]" in src and "gt_add<2>" in src
    assert "gt_find_or_insert_pre<uint32_t>" in src  # first buckets of all rows loaded ahead


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


def test_split_batch_counts():
    """vc_batch_new_split leaves queries whose largest pipeline reaches solo_rows out of the
    persistent kernel."""
    from vldb_voila_b200.engine import Batch
    specs = ["sel_aggr:rows=1000", "sel_aggr:rows=200000", "groupby:rows=5000,keys=100", "star:rows=300000"]
    engines, queries = [], []
    for s in specs:
        w, e = offline(s)
        engines.append(e)
        queries.append(e.query(w.plan))
    info = Batch(queries, solo_rows=100000).info()
    assert (info["queries"], info["batched"], info["solo"]) == (4, 2, 2)
    assert Batch(queries).info()["solo"] == 0
    assert Batch(queries, solo_rows=1).info()["work_items"] == 0


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
    # a build side that is itself a join: its build items must wait for the inner build
    queries.append(engines[-3].query(NESTED_BUILD_PLAN))
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
    # the nested query (last): date build, then the customer build that probes it, then the
    # fact pipeline -- three distinct done-counters chained by their waits
    nested = [r for r in work if r[F["params"]] >= sorted(set(work[:, F["params"]]))[-3]]
    done_counters = []
    for r in nested:
        if r[F["done"]] not in done_counters:
            done_counters.append(r[F["done"]])
    assert len(done_counters) == 3, done_counters
    by_done = {d: [r for r in nested if r[F["done"]] == d] for d in done_counters}
    assert all(r[F["dep"]] == done_counters[0] for r in by_done[done_counters[1]])
    assert all(r[F["dep"]] == done_counters[1] for r in by_done[done_counters[2]])


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


@pytest.mark.parametrize("flavor", ["cuda(rows=3)", "cuda(threads=100)", "cuda(aggr=magic)", "gpu(x=1)", "cuda(nokey=1)",
                                    "cuda(lowcard=stacked)", "cuda(minctas=33)", "cuda(minctas=-1)", "cuda(pgroups=17)",
                                    "cuda(stream=cg)"])
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


JOIN_N_PLAN = ("(aggr hash ((col customer.c_region)) ((fun sum (col lineorder.lo_revenue)) (fun count))"
               " (join joinN ((col customer.c_custkey)) () (scan customer (c_custkey c_region))"
               " ((col lineorder.lo_custkey)) ((col lineorder.lo_revenue)) (scan lineorder (lo_custkey lo_revenue))))")


@pytest.mark.parametrize("flavor", FLAVORS)
def test_join_n_plans_compile(flavor):
    """JoinN probes: a hash table (never dense: duplicates need their own slots) and a match
    loop around the rest of the pipeline."""
    w, e = offline("star:rows=1000,custs=50")
    q = e.query(JOIN_N_PLAN, flavor)
    src = q.source()
    assert "__any_sync" in src and "1ull) * SPB" in src  # the match loop may walk the whole table
    assert "vd::dense_test" not in src


def test_join_n_rejects_dense_builds():
    w, e = offline("star:rows=1000,custs=50")
    with pytest.raises(VoilaError) as ex:
        e.query(JOIN_N_PLAN, "cuda(build=dense)")
    assert ex.value.code == 6


def test_sub_aggregation_lowers_to_an_intermediate_table():
    """An aggregation below the root writes an intermediate table that the next pipeline scans
    (row count read on the device); its columns carry the reference translator's names."""
    from helpers import manifest
    m = manifest()["agg_of_agg"]
    w, e = offline(m["spec"])
    q = e.query(m["plan"])
    info = q.info()
    assert [p["sink"] for p in info["pipelines"]] == ["aggr_dense", "aggr_hash"]
    src = q.source()
    assert "__ldcg(((const unsigned long long*)" in src  # the consumer's row count
    # a join takes the translator's next id before its build side: below it, the first
    # aggregation's table is aggr_ht2, and aggr_ht1 names nothing
    plan = ("(aggr global () ((fun count)) (join join01 ((col X.key_0)) ()"
            " (aggr hash ((col lineitem.l_orderkey)) ((fun count)) (scan lineitem (l_orderkey)))"
            " ((col lineitem.l_orderkey)) () (scan lineitem (l_orderkey))))")
    e.query(plan.replace("X", "aggr_ht2"))
    with pytest.raises(VoilaError) as ex:
        e.query(plan.replace("X", "aggr_ht1"))
    assert ex.value.code == 1


def test_sub_aggregations_are_not_batched_yet():
    from helpers import manifest
    from vldb_voila_b200.engine import Batch
    m = manifest()["having_global"]
    w, e = offline(m["spec"])
    with pytest.raises(VoilaError) as ex:
        Batch([e.query(m["plan"])])
    assert ex.value.code == 6


def test_sums_beyond_int64_are_split_into_exact_chunk_sums():
    """sum(w) over 40,000 values up to 2e15 can reach 8e19: it is computed as int64 sums of bit
    chunks of w (recombined in 128 bits on the host), never rejected and never wrapped."""
    w, e = offline("bigsum:rows=40000,seed=95")
    q = e.query(w.plan)
    src = q.source()
    assert "& 1073741823ull" in src or "ull))" in src
    assert ">> " in src
    info = q.info()
    # physical result columns: key, sum(v) in 2 chunks, sum(w) in 2 chunks, count
    assert info["result_cols"] == 6
    # a sub-aggregation cannot hand 128-bit values to a later pipeline: rejected, not wrapped
    plan = ("(aggr global () ((fun count)) (select (fun > (col aggr_ht1.aggr_0) (const 0))"
            " (aggr hash ((col fact.g)) ((fun sum (col fact.w))) (scan fact (g w)))))")
    with pytest.raises(VoilaError) as ex:
        e.query(plan)
    assert ex.value.code == 6


def test_per_pipeline_flavor_overrides():
    """"cuda(...);p<id>=cuda(...)" gives single pipelines their own knobs (the reference's
    per-pipeline blends); hash and graph stay query-wide."""
    w, e = offline("star:rows=1000")
    q = e.query(w.plan, "cuda(threads=256);p4=cuda(rows=8,threads=128);p1=cuda(build=staged)")
    info = q.info()
    assert info["flavor"].endswith(";p4=cuda(rows=8,threads=128);p1=cuda(build=staged)")
    ks = {k["name"]: k["threads"] for k in info["kernels"]}
    assert ks["vc_p4_main"] == 128 and ks["vc_p3_main"] == 256
    assert "vc_p1_insert" in ks and "vc_p2_insert" not in ks
    for bad in ["cuda();p4=cuda(hash=voila)", "cuda();q4=cuda(rows=2)", "cuda();p4=cuda(rows=3)"]:
        with pytest.raises(VoilaError):
            e.query(w.plan, bad)


def test_partitioned_aggregation_plan():
    """aggr=part: a histogram pass counts each partition's rows per CTA, the pipeline's kernel
    (same grid, same tiles per CTA) writes each record at its partition's next position, so
    every partition's records are contiguous, and a persistent kernel aggregates each
    partition in shared memory and writes its result rows itself (no group table, no
    extraction scan)."""
    w, e = offline("groupby:rows=6000000,keys=1500000,zipf=0,seed=3")
    q = e.query(w.plan, "cuda(aggr=part)")
    src = q.source()
    info = q.info()
    # 2 x 1.5M groups / 4096 slots per partition table -> 1024 partitions
    assert "vd::block_excl_scan(stot, shist, 1024" in src and "atomicAdd(&scur[" in src
    assert "vd::st_find_or_insert(skeys, 4096" in src and "gt_find_or_insert" not in src
    k = {x["name"]: x for x in info["kernels"]}
    assert [x["name"] for x in info["kernels"]] == ["vc_p0_hist", "vc_p0_main", "vc_p0_extract"]
    assert k["vc_p0_extract"]["threads"] == 512 and k["vc_p0_hist"]["smem"] == 1024 * 8
    # the scatter pass keeps one cursor per partition in shared memory
    assert k["vc_p0_main"]["smem"] == 1024 * 4
    # the histogram pass reads the key column only
    hist = src[src.index("vc_p0_hist"):src.index("vc_p0_main")]
    assert "load_rows<int32_t, 4>(c0" in hist and "(c1" not in hist and "(c2" not in hist
    # an explicit partition count
    src2 = e.query(w.plan, "cuda(aggr=part,parts=2048,threads=512)").source()
    assert "vd::block_excl_scan(stot, shist, 2048" in src2
    # too few partitions for the groups bound: falls back to the global table
    assert "gt_find_or_insert" in e.query(w.plan, "cuda(aggr=part,parts=16)").source()
    # aggr=auto: a key space no larger than the hash table would be takes the direct table
    # (slot = packed key); a wider one with more than 2^18 groups is partitioned, fewer
    # groups take the hash table
    auto = e.query(w.plan).source()
    assert "_hist" not in auto and "gt_find_or_insert" not in auto and "gt_cache_add" in auto
    wide = ("(aggr hash ((col k)) ((fun sum (col lineitem.l_extendedprice)) (fun count)) (project ((assign k "
            "(fun * (col lineitem.l_orderkey) (const 1000))) (col lineitem.l_extendedprice)) "
            "(scan lineitem (l_orderkey l_extendedprice))))")
    assert "_hist" in e.query(wide).source()
    w2, e2 = offline("groupby:rows=100000,keys=200000,zipf=0,seed=3")
    src3 = e2.query(wide).source()
    assert "_hist" not in src3 and "gt_find_or_insert" in src3


@pytest.mark.parametrize("flavor", ["cuda(parts=24)", "cuda(parts=8)", "cuda(parts=4096)", "cuda(frows=3)", "cuda(frows=32)"])
def test_bad_partition_knobs_are_rejected(flavor):
    w, e = offline("groupby:rows=1000,keys=100000")
    with pytest.raises(VoilaError) as ex:
        e.query(w.plan, flavor)
    assert ex.value.code == 1


def test_batched_partitioned_aggregation_uses_a_group_table():
    """A batch runs a query prepared with aggr=part through the global group table."""
    from vldb_voila_b200.engine import Batch
    w, e = offline("groupby:rows=100000,keys=100000")
    q = e.query(w.plan, "cuda(aggr=part)")
    assert "_hist" in q.source()
    b = Batch([q])
    src = b.source()
    assert "gt_find_or_insert" in src and "scur" not in src


def test_direct_group_table_plan():
    """aggr=auto over a key space no larger than the hash table: the accumulator words are indexed
    by the packed key (no stored keys, no probes) behind the shared-memory cache; aggr=direct drops
    the cache; a key space of 2^28 slots and more keeps the hash table."""
    w, e = offline("groupby:rows=6000000,keys=1500000,zipf=0,seed=3")
    auto = e.query(w.plan).source()
    assert "gt_add<2>(gacc, (int64_t)pk, w)" in auto and "gt_cache_add" in auto
    assert "gt_find_or_insert" not in auto and "gkeys" not in auto
    direct = e.query(w.plan, "cuda(aggr=direct)").source()
    assert "gt_cache_add" not in direct and "gt_add<2>(gacc, (int64_t)pk, w)" in direct
    # the extraction loads every word of its chunk before clearing any slot, and reserves rows per warp
    ext = direct[direct.index("_extract("):]
    assert ext.index("__ldcg(&gacc[") < ext.index("= 0ull; }") and "__ballot_sync" in ext
    wide = ("(aggr hash ((col k)) ((fun count)) (project ((assign k (fun * (col lineitem.l_orderkey) "
            "(const 1000)))) (scan lineitem (l_orderkey))))")
    w2, e2 = offline("groupby:rows=100000,keys=1000000,zipf=0,seed=3")
    assert "gt_find_or_insert" in e2.query(wide, "cuda(aggr=direct)").source()


def test_packed_low_cardinality_accumulators():
    """lowcard=packed (the default): per-thread packed words per block-dictionary code in shared
    memory, folded per warp by redux.sync; it falls back to warp pre-combining where its words
    would take more than 64 KiB per CTA, and under survivor compaction (the star chain)."""
    w, e = offline("sel_aggr:rows=6000000,seed=1")
    src = e.query(w.plan).source()
    assert "racc(code, 0) +=" in src and "rflush();" in src and "vd::group_sum_u<" in src
    assert "warp_combine" not in src
    assert "warp_combine" in e.query(w.plan, "cuda(threads=1024)").source()
    regs = e.query(w.plan, "cuda(lowcard=regs)").source()
    assert "racc_r[" in regs and "code == k ?" in regs
    ws, es = offline("star:rows=100000")
    assert "racc(" not in es.query(ws.plan).source()


def test_tma_ring_without_block_barriers():
    """load=tma: a warp-only body (no block collectives) takes the ring with per-stage empty
    barriers that every warp arrives on; an appending sink keeps the ring with a block barrier
    per tile."""
    w, e = offline("sel_aggr:rows=100000")
    src = e.query(w.plan, "cuda(load=tma,stages=3)").source()
    assert "vd::mbar_arrive(&empty[s])" in src and "vd::mbar_init(&empty[s], 8)" in src
    assert "__any_sync(0xffffffffu, !ok" in src
    emit = ("(select (fun <= (col lineitem.l_shipdate) (const 9000)) "
            "(scan lineitem (l_shipdate l_quantity)))")
    src2 = e.query(emit, "cuda(load=tma,stages=2)").source()
    assert "empty[" not in src2 and "vd::block_any(!ok)" in src2


def test_stream_noalloc_loads_columns_without_l1_allocation():
    """stream=noalloc: every column load of the fused kernel (eager tiles and the compaction
    flush's gathers) takes load mode 2 (ld.global.nc.L1::no_allocate); the default keeps the
    read-only path."""
    w, e = offline("star:rows=100000")
    src = e.query(w.plan, "cuda(stream=noalloc)").source()
    main = src[src.index("vc_p4_main"):]
    assert "vd::load_rows<int32_t, 4, 2>(c0" in main and "vd::load_one<int32_t, 2>(" in main
    assert ", 2>(" not in e.query(w.plan).source()
    assert "stream=noalloc" in e.query(w.plan, "cuda(stream=noalloc)").info()["flavor"]
