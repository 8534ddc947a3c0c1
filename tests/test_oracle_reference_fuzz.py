"""The oracle against the reference itself on seeded random plans: selections, projections,
hash, global and emitting roots over the lineitem-shaped table, Join01 probe chains over the star
schema, JoinN joins, aggregations over aggregations, string predicates and keys, sums past int64
and extract_year keys.  Each plan runs through the reference's vectorwise flavor, built from its sources
by oracle/ref/Makefile, and through the oracle, and the sorted result lines must be identical.
CPU only; skipped where the reference build or its source tree is absent."""
import os
import subprocess
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle.voila_oracle import result_lines, run_plan
from vldb_voila_b200 import generate_workload_host, workload

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("VOILA_REFERENCE", "/root/reference")
RDIR = os.path.join(REPO, "oracle", "_ref", "avx512")
SPEC = "sel_aggr:rows=20000,seed=81"
N_PLANS = 16

# the workload's columns and their value ranges (sel_aggr generator)
COLS = {"l_quantity": (1, 50), "l_extendedprice": (90000, 10500000), "l_discount": (0, 10), "l_tax": (0, 8),
        "l_returnflag": (65, 82), "l_linestatus": (70, 79), "l_shipdate": (2448623, 2451148)}
SMALL = ["l_quantity", "l_discount", "l_tax", "l_returnflag", "l_linestatus"]
# the flag columns' values ({A,N,R}, {F,O}): equality constants mostly hit one of them
FLAGS = {"l_returnflag": [65, 78, 82], "l_linestatus": [70, 79]}


def _have_reference():
    if not (os.path.isdir(REF) and os.path.exists(os.path.join(RDIR, "ref_gen"))):
        return False
    with open("/proc/cpuinfo") as f:
        return "avx512f" in f.read()


def _col(name):
    return f"(col lineitem.{name})" if name in COLS else f"(col {name})"


def _predicate(rng):
    parts = []
    for _ in range(int(rng.integers(1, 4))):
        c = str(rng.choice(list(COLS)))
        lo, hi = COLS[c]
        op = str(rng.choice(["<", "<=", ">", ">=", "=", "!="]))
        v = int(rng.integers(lo, hi + 1))
        if c in FLAGS and rng.random() < 0.8:
            v = int(rng.choice(FLAGS[c]))
        parts.append(f"(fun {op} {_col(c)} (const {v}))")
    expr = parts[0]
    for p in parts[1:]:
        expr = f"(fun {rng.choice(['and', 'or'])} {expr} {p})"
    return expr


def _derived(rng):
    """One projected column: its plan expression and whether its range is small enough for a key."""
    k = int(rng.integers(1, 30))
    choices = [
        (f"(fun - (col lineitem.l_extendedprice) (fun * (col lineitem.l_quantity) (const {k * 1000})))", False),
        ("(fun * (col lineitem.l_quantity) (col lineitem.l_discount))", True),
        (f"(fun + (col lineitem.l_tax) (const {k}))", True),
        (f"(fun - (const {k}) (col lineitem.l_discount))", True),
    ]
    return choices[int(rng.integers(0, len(choices)))]


def random_plan(seed):
    rng = np.random.default_rng(seed)
    scan = "(scan lineitem (" + " ".join(COLS) + "))"
    src = f"(select {_predicate(rng)} {scan})" if rng.random() < 0.8 else scan
    kind = str(rng.choice(["hash", "hash", "global", "emit"]))
    if kind == "emit":
        return f"(select {_predicate(rng)} {scan})"
    dexpr, dsmall = _derived(rng)
    proj = "(project ((assign x1 " + dexpr + ") " + " ".join(_col(c) for c in COLS) + ") " + src + ")"
    sums = [str(c) for c in rng.choice(["l_extendedprice", "l_quantity", "x1", "l_discount"],
                                       size=int(rng.integers(1, 4)), replace=False)]
    aggs = " ".join(f"(fun sum {_col(c)})" for c in sums)
    if kind == "global":
        return f"(aggr global () ({aggs} (fun count)) {proj})"
    keypool = SMALL + (["x1"] if dsmall else [])
    keys = [str(c) for c in rng.choice(keypool, size=int(rng.integers(1, 3)), replace=False)]
    count = " (fun count)" if rng.random() < 0.7 else ""
    return f"(aggr hash ({' '.join(_col(c) for c in keys)}) ({aggs}{count}) {proj})"


def _reference_results(jobs, tmp):
    """Sorted result lines of each (tag, plan, spec) job from the reference's vectorwise flavor:
    the query libraries are generated and compiled in parallel, then run one after another."""
    gen, run = os.path.join(RDIR, "ref_gen"), os.path.join(RDIR, "ref_run")
    cxx = (f"g++ -march=skylake-avx512 -mtune=generic -O3 -g0 -std=c++17 -include cstdint -DIS_RELEASE -w "
           f"-I{REPO}/oracle/ref/shim -I{RDIR}/gen -I{REF} -I{REF}/libs -I{REF}/db-engine-paradigms/include")

    def build(job):
        tag, plan, spec = job
        lib = os.path.join(tmp, f"{tag}.so")
        r = subprocess.run([gen, "--workload", spec, "--flavor", "vectorwise", "--out", lib, "--cxx", cxx,
                            "--plan", plan], capture_output=True, text=True)
        return lib, r

    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as pool:
        built = list(pool.map(build, jobs))
    out = {}
    for (tag, plan, spec), (lib, r) in zip(jobs, built):
        assert r.returncode == 0, (plan, r.stderr[-2000:])
        res = os.path.join(tmp, f"{tag}.txt")
        r = subprocess.run([run, "--workload", spec, "--lib", lib, "--flavor", "vectorwise", "--threads", "4",
                            "--reps", "1", "--result", res], capture_output=True, text=True)
        assert r.returncode == 0, (plan, r.stderr[-2000:])
        out[tag] = sorted(line for line in open(res).read().split("\n") if line)
    return out


def _check(jobs, data_of):
    with tempfile.TemporaryDirectory() as tmp:
        expect = _reference_results(jobs, tmp)
    for tag, plan, spec in jobs:
        assert result_lines(run_plan(plan, data_of[spec])) == expect[tag], plan


@pytest.mark.skipif(not _have_reference(), reason="needs the reference build (oracle/_ref) and its source tree")
def test_oracle_matches_reference_on_random_plans():
    _check([(f"p{i}", random_plan(1000 + i), SPEC) for i in range(N_PLANS)],
           {SPEC: generate_workload_host(workload(SPEC))})


def test_random_plans_are_deterministic_and_varied():
    plans = [random_plan(1000 + i) for i in range(N_PLANS)]
    assert plans == [random_plan(1000 + i) for i in range(N_PLANS)]
    roots = {p.split(" ")[0] + " " + p.split(" ")[1] for p in plans}
    assert {"(aggr hash", "(aggr global", "(select (fun"} <= roots


STAR_SPEC = "star:rows=20000,dates=300,custs=500,supps=20,parts=400,seed=83"
N_JOIN_PLANS = 10
# dimension: (fact foreign key, dimension key, attributes with their ranges)
DIMS = {"date": ("lo_orderdate", "d_datekey", {"d_year": (1992, 1998), "d_weekday": (0, 6)}),
        "customer": ("lo_custkey", "c_custkey", {"c_region": (0, 4), "c_mktsegment": (0, 4)}),
        "part": ("lo_partkey", "p_partkey", {"p_category": (0, 24)})}
FACT = "(scan lineorder (lo_orderdate lo_custkey lo_suppkey lo_partkey lo_revenue lo_supplycost))"


def random_join_plan(seed):
    """A probe chain of one to three Join01 joins of the fact table with filtered dimensions, a
    root grouped by dimension attributes (or global), summing fact columns."""
    rng = np.random.default_rng(seed)
    cur = FACT
    if rng.random() < 0.4:
        cur = f"(select (fun < (col lineorder.lo_revenue) (const {int(rng.integers(1, 10_000_000))})) {cur})"
    dims = [str(d) for d in rng.choice(list(DIMS), size=int(rng.integers(1, 4)), replace=False)]
    attrs = []
    for d in dims:
        fk, key, cols = DIMS[d]
        a = str(rng.choice(list(cols)))
        attrs.append(f"{d}.{a}")
        src = f"(scan {d} ({key} {' '.join(cols)}))"
        if rng.random() < 0.7:
            c = str(rng.choice(list(cols)))
            lo, hi = cols[c]
            op = str(rng.choice(["<", "<=", ">=", "=", "!="]))
            src = f"(select (fun {op} (col {d}.{c}) (const {int(rng.integers(lo, hi + 1))})) {src})"
        cur = f"(join join01 ((col lineorder.{fk})) () {cur} ((col {d}.{key})) ((col {d}.{a})) {src})"
    sums = "(fun sum (col lineorder.lo_revenue))"
    if rng.random() < 0.5:
        sums += " (fun sum (col lineorder.lo_supplycost))"
    if rng.random() < 0.25:
        return f"(aggr global () ({sums} (fun count)) {cur})"
    keys = [str(a) for a in rng.choice(attrs, size=int(rng.integers(1, len(attrs) + 1)), replace=False)]
    return f"(aggr hash ({' '.join(f'(col {k})' for k in keys)}) ({sums} (fun count)) {cur})"


@pytest.mark.skipif(not _have_reference(), reason="needs the reference build (oracle/_ref) and its source tree")
def test_oracle_matches_reference_on_random_join_plans():
    _check([(f"j{i}", random_join_plan(2000 + i), STAR_SPEC) for i in range(N_JOIN_PLANS)],
           {STAR_SPEC: generate_workload_host(workload(STAR_SPEC))})


N_NESTED_PLANS = 8


def random_nested_plan(seed):
    """JoinN (the fact table as the build side, so every key has many matches) or an aggregation
    over an aggregation (the inner one's outputs named aggr_ht1.key_<i> / aggr_ht1.aggr_<j>, as
    the reference's translator names them)."""
    rng = np.random.default_rng(seed)
    if rng.random() < 0.5:
        d = str(rng.choice(["customer", "date"]))
        fk, key, cols = DIMS[d]
        a = str(rng.choice(list(cols)))
        src = f"(scan {d} ({key} {' '.join(cols)}))"
        if rng.random() < 0.6:
            lo, hi = cols[a]
            src = f"(select (fun <= (col {d}.{a}) (const {int(rng.integers(lo, hi + 1))})) {src})"
        pay = str(rng.choice(["lo_revenue", "lo_supplycost"]))
        join = (f"(join joinN ((col {d}.{key})) () {src} ((col lineorder.{fk})) ((col lineorder.{pay})) "
                f"(scan lineorder ({fk} {pay})))")
        return f"(aggr hash ((col {d}.{a})) ((fun sum (col lineorder.{pay})) (fun count)) {join})"
    k = str(rng.choice(["l_quantity", "l_discount", "l_tax"]))
    v = str(rng.choice(["l_extendedprice", "l_quantity"]))
    inner = (f"(aggr hash ((col lineitem.{k}) (col lineitem.l_returnflag)) ((fun sum (col lineitem.{v})) (fun count)) "
             f"(scan lineitem ({k} l_returnflag {v})))")
    if rng.random() < 0.5:
        return f"(aggr hash ((col aggr_ht1.key_1)) ((fun sum (col aggr_ht1.aggr_0)) (fun count)) {inner})"
    return (f"(aggr global () ((fun sum (col aggr_ht1.aggr_1)) (fun count)) "
            f"(select (fun > (col aggr_ht1.aggr_1) (const {int(rng.integers(100, 700))})) {inner}))")


@pytest.mark.skipif(not _have_reference(), reason="needs the reference build (oracle/_ref) and its source tree")
def test_oracle_matches_reference_on_random_nested_plans():
    plans = [random_nested_plan(3000 + i) for i in range(N_NESTED_PLANS)]
    _check([(f"n{i}", p, STAR_SPEC if "joinN" in p else SPEC) for i, p in enumerate(plans)],
           {STAR_SPEC: generate_workload_host(workload(STAR_SPEC)), SPEC: generate_workload_host(workload(SPEC))})


STR_SPEC = "strings:rows=20000,parts=600,seed=84"
N_STRING_PLANS = 10
PATTERNS = ["re", "ee", "pink", "a", "zz", "ol", "white", "navy"]
BRANDS = ["azure", "black", "amber", "coral", "none"]


def random_string_plan(seed):
    """Predicates on string columns (contains on p_name, equality on p_brand) under and/or, for an
    emitting select over the string table or a join grouped by a string key."""
    rng = np.random.default_rng(seed)
    parts = []
    for _ in range(int(rng.integers(1, 3))):
        if rng.random() < 0.6:
            parts.append(f"(fun contains (col part.p_name) (const {rng.choice(PATTERNS)}))")
        else:
            parts.append(f"(fun {rng.choice(['=', '!='])} (col part.p_brand) (const {rng.choice(BRANDS)}))")
    pred = parts[0]
    for p in parts[1:]:
        pred = f"(fun {rng.choice(['and', 'or'])} {pred} {p})"
    part = f"(select {pred} (scan part (p_partkey p_name p_brand)))"
    if rng.random() < 0.25:
        return part
    key = str(rng.choice(["p_brand", "p_name"]))
    return (f"(aggr hash ((col part.{key})) ((fun sum (col lineitem.l_extendedprice)) (fun count)) "
            f"(join join01 ((col lineitem.l_partkey)) () (scan lineitem (l_partkey l_extendedprice)) "
            f"((col part.p_partkey)) ((col part.{key})) {part}))")


@pytest.mark.skipif(not _have_reference(), reason="needs the reference build (oracle/_ref) and its source tree")
def test_oracle_matches_reference_on_random_string_plans():
    _check([(f"s{i}", random_string_plan(4000 + i), STR_SPEC) for i in range(N_STRING_PLANS)],
           {STR_SPEC: generate_workload_host(workload(STR_SPEC))})


WIDE_SPEC = "bigsum:rows=40000,seed=85"
N_WIDE_PLANS = 6


def random_wide_plan(seed):
    """Sums whose bound leaves int64 (values up to ±2e15 over 40,000 rows: the reference types them
    i128), grouped or global, behind a filter on the group column or the values; and extract_year
    keys over the lineitem-shaped table."""
    rng = np.random.default_rng(seed)
    if rng.random() < 0.3:
        d = int(rng.integers(2448623, 2451148))
        return (f"(aggr hash ((col y)) ((fun sum (col lineitem.l_quantity)) (fun count)) (project ((assign y (fun "
                f"extract_year (col lineitem.l_shipdate))) (col lineitem.l_quantity)) (select (fun >= "
                f"(col lineitem.l_shipdate) (const {d})) (scan lineitem (l_shipdate l_quantity)))))")
    sums = " ".join(f"(fun sum (col fact.{c}))" for c in rng.choice(["v", "w"], size=int(rng.integers(1, 3)), replace=False))
    if rng.random() < 0.5:
        src = f"(select (fun != (col fact.g) (const {int(rng.integers(0, 4))})) (scan fact (g v w)))"
    else:
        src = f"(select (fun > (col fact.v) (const {int(rng.integers(-10**15, 10**15))})) (scan fact (g v w)))"
    if rng.random() < 0.4:
        return f"(aggr global () ({sums} (fun count)) {src})"
    return f"(aggr hash ((col fact.g)) ({sums} (fun count)) {src})"


@pytest.mark.skipif(not _have_reference(), reason="needs the reference build (oracle/_ref) and its source tree")
def test_oracle_matches_reference_on_random_wide_and_year_plans():
    plans = [random_wide_plan(5000 + i) for i in range(N_WIDE_PLANS)]
    _check([(f"w{i}", p, SPEC if "extract_year" in p else WIDE_SPEC) for i, p in enumerate(plans)],
           {WIDE_SPEC: generate_workload_host(workload(WIDE_SPEC)), SPEC: generate_workload_host(workload(SPEC))})
