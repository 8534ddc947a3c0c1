"""Regenerates the golden result fixtures from the reference itself.

Runs the reference's hyper and vectorwise flavors (compiled from the reference sources by
oracle/ref/Makefile into oracle/_ref/<isa>/; needs the reference tree, so it runs on the
build host only) on seeded synthetic workloads and stores their sorted QueryResult lines as
tests/golden/<case>.<flavor>.txt, plus manifest.json with each case's workload spec, plan
and the reference loader's data checksum.

    python tests/golden/make_golden.py [--isa avx512]
"""
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("VOILA_REFERENCE", "/root/reference")

SEL_EMIT = ("(select (fun < (col lineitem.l_quantity) (const 3))"
            " (scan lineitem (l_quantity l_discount l_returnflag)))")
Q6_GLOBAL = ("(aggr global () ((fun sum (fun * (col lineitem.l_extendedprice) (col lineitem.l_discount))) (fun count))"
             " (select (fun and (fun and (fun >= (col lineitem.l_discount) (const 5)) (fun <= (col lineitem.l_discount) (const 7)))"
             " (fun < (col lineitem.l_quantity) (const 24)))"
             " (scan lineitem (l_extendedprice l_discount l_quantity))))")
NEG_KEYS = ("(aggr hash ((col qk)) ((fun sum (col neg)) (fun count))"
            " (project ((assign qk (fun - (col lineitem.l_quantity) (const 25)))"
            " (assign neg (fun - (col lineitem.l_tax) (col lineitem.l_extendedprice))))"
            " (select (fun or (fun = (col lineitem.l_returnflag) (const 65)) (fun != (col lineitem.l_linestatus) (const 79)))"
            " (scan lineitem (l_quantity l_tax l_extendedprice l_returnflag l_linestatus)))))")
JOIN_N = ("(aggr hash ((col customer.c_region)) ((fun sum (col lineorder.lo_revenue)) (fun count))"
          " (join joinN ((col customer.c_custkey)) () (scan customer (c_custkey c_region))"
          " ((col lineorder.lo_custkey)) ((col lineorder.lo_revenue)) (scan lineorder (lo_custkey lo_revenue))))")
JOIN_2KEY = ("(aggr hash ((col customer.c_mktsegment)) ((fun sum (col lineorder.lo_supplycost)) (fun count))"
             " (join join01 ((col lineorder.lo_custkey) (col lineorder.lo_partkey)) ()"
             " (scan lineorder (lo_custkey lo_partkey lo_supplycost))"
             " ((col customer.c_custkey) (col customer.c_custkey)) ((col customer.c_mktsegment))"
             " (scan customer (c_custkey c_mktsegment))))")
JOIN_EMIT = ("(select (fun = (col date.d_year) (const 1995))"
             " (join join01 ((col lineorder.lo_orderdate)) () (scan lineorder (lo_orderdate lo_revenue))"
             " ((col date.d_datekey)) ((col date.d_year)) (scan date (d_datekey d_year))))")

# aggregation below the plan root: the sub-aggregation's outputs are named
# aggr_ht<N>.key_<i> / aggr_ht<N>.aggr_<j> by the reference's translator
AGG_OF_AGG = ("(aggr hash ((col aggr_ht1.aggr_1)) ((fun sum (col aggr_ht1.aggr_0)) (fun count))"
              " (aggr hash ((col lineitem.l_orderkey)) ((fun sum (col lineitem.l_quantity)) (fun count))"
              " (scan lineitem (l_orderkey l_quantity))))")
HAVING_GLOBAL = ("(aggr global () ((fun sum (col aggr_ht1.aggr_0)) (fun count))"
                 " (select (fun > (col aggr_ht1.aggr_1) (const 10))"
                 " (aggr hash ((col lineitem.l_orderkey)) ((fun sum (col lineitem.l_extendedprice)) (fun count))"
                 " (scan lineitem (l_orderkey l_extendedprice)))))")
HAVING_EMIT = ("(select (fun > (col aggr_ht1.aggr_0) (const 200))"
               " (aggr hash ((col lineitem.l_orderkey)) ((fun sum (col lineitem.l_quantity)))"
               " (scan lineitem (l_orderkey l_quantity))))")

# sums whose bound leaves int64: the reference types them i128
WIDE_GLOBAL = ("(aggr global () ((fun sum (col fact.w)) (fun sum (col fact.v)) (fun count))"
               " (scan fact (v w)))")

YEARS = ("(aggr hash ((col y) (col lineitem.l_returnflag)) ((fun sum (col lineitem.l_quantity)) (fun count))"
         " (project ((assign y (fun extract_year (col lineitem.l_shipdate))) (col lineitem.l_returnflag)"
         " (col lineitem.l_quantity)) (scan lineitem (l_shipdate l_returnflag l_quantity))))")

# string columns: a string equality filter emitting strings, and string group keys
STR_EMIT = ("(select (fun and (fun = (col part.p_brand) (const coral)) (fun contains (col part.p_name) (const red)))"
            " (scan part (p_partkey p_name p_brand)))")
STR_GROUP = ("(aggr hash ((col part.p_name)) ((fun count)) (select (fun != (col part.p_brand) (const amber))"
             " (scan part (p_name p_brand))))")

CASES = [
    ("sel_aggr_1k", "sel_aggr:rows=1000,seed=11", None),
    ("sel_aggr_100k", "sel_aggr:rows=100000,seed=12", None),
    ("sel_aggr_tiny_sel", "sel_aggr:rows=5000,sel=0.002,seed=13", None),
    ("sel_aggr_all", "sel_aggr:rows=20000,sel=1,seed=14", None),
    ("join_aggr_small", "join_aggr:build=20000,probe=100000,seed=21", None),
    ("join_aggr_sel1", "join_aggr:build=5000,probe=20000,sel=1,seed=22", None),
    ("join_aggr_nomatch", "join_aggr:build=5000,probe=20000,sel=0,seed=23", None),
    ("groupby_uniform", "groupby:rows=100000,keys=2000,zipf=0,seed=31", None),
    ("groupby_zipf125", "groupby:rows=100000,keys=2000,zipf=1.25,seed=32", None),
    ("groupby_zipf05", "groupby:rows=50000,keys=3000,zipf=0.5,seed=34", None),
    ("groupby_one_key", "groupby:rows=10000,keys=1,seed=33", None),
    ("star_small", "star:rows=100000,custs=3000,supps=200,parts=14000,seed=41", None),
    ("star_tiny", "star:rows=3000,dates=200,custs=50,supps=20,parts=300,seed=42", None),
    ("select_emit", "sel_aggr:rows=2000,seed=51", SEL_EMIT),
    ("q6_global", "sel_aggr:rows=50000,seed=52", Q6_GLOBAL),
    ("neg_keys", "sel_aggr:rows=30000,seed=53", NEG_KEYS),
    ("join_n", "star:rows=20000,dates=100,custs=500,supps=10,parts=100,seed=54", JOIN_N),
    ("join_2key", "star:rows=20000,dates=100,custs=500,supps=10,parts=400,seed=55", JOIN_2KEY),
    ("join_emit", "star:rows=5000,dates=2556,custs=10,supps=10,parts=10,seed=56", JOIN_EMIT),
    ("agg_of_agg", "groupby:rows=20000,keys=3000,zipf=0.8,seed=71", AGG_OF_AGG),
    ("having_global", "groupby:rows=20000,keys=3000,zipf=0.8,seed=72", HAVING_GLOBAL),
    ("having_emit", "groupby:rows=20000,keys=3000,zipf=0.8,seed=73", HAVING_EMIT),
    ("wide_sums", "bigsum:rows=40000,seed=95", None),
    ("wide_global", "bigsum:rows=40000,seed=96", WIDE_GLOBAL),
    ("extract_year", "sel_aggr:rows=30000,seed=57", YEARS),
    ("strings_contains", "strings:rows=50000,parts=3000,seed=58", None),
    ("strings_emit", "strings:rows=1000,parts=4000,seed=59", STR_EMIT),
    ("strings_group", "strings:rows=1000,parts=5000,seed=60", STR_GROUP),
]


def main():
    isa = "avx512"
    if "--isa" in sys.argv:
        isa = sys.argv[sys.argv.index("--isa") + 1]
    rdir = os.path.join(REPO, "oracle", "_ref", isa)
    gen, run = os.path.join(rdir, "ref_gen"), os.path.join(rdir, "ref_run")
    march = "-march=skylake-avx512" if isa == "avx512" else "-march=haswell"
    cxx = (f"g++ {march} -mtune=generic -O3 -g0 -std=c++17 -include cstdint -DIS_RELEASE -w "
           f"-I{REPO}/oracle/ref/shim -I{rdir}/gen -I{REF} -I{REF}/libs -I{REF}/db-engine-paradigms/include")
    manifest = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, spec, plan in CASES:
            entry = {"spec": spec, "plan": plan}
            for flavor in ("hyper", "vectorwise"):
                lib = os.path.join(tmp, f"{name}_{flavor}.so")
                cmd = [gen, "--workload", spec, "--flavor", flavor, "--out", lib, "--cxx", cxx]
                if plan:
                    cmd += ["--plan", plan]
                r = subprocess.run(cmd, capture_output=True, text=True)
                if r.returncode != 0:
                    print(name, flavor, "generation failed", r.stderr[-2000:])
                    entry[flavor] = {"status": "generate_failed"}
                    continue
                res = os.path.join(tmp, f"{name}_{flavor}.txt")
                r = subprocess.run([run, "--workload", spec, "--lib", lib, "--flavor", flavor, "--threads", "4",
                                    "--reps", "1", "--result", res, "--checksum", "1"],
                                   capture_output=True, text=True)
                if r.returncode != 0:
                    print(name, flavor, "run failed", r.returncode, r.stderr[-2000:])
                    entry[flavor] = {"status": f"run_failed_{r.returncode}"}
                    continue
                info = json.loads(r.stdout.strip().splitlines()[-1])
                lines = sorted(l for l in open(res).read().split("\n") if l)
                with open(os.path.join(HERE, f"{name}.{flavor}.txt"), "w") as f:
                    f.write("\n".join(lines) + ("\n" if lines else ""))
                entry[flavor] = {"status": "ok", "rows": len(lines)}
                entry["checksum"] = str(info.get("checksum"))
                print(name, flavor, len(lines), "rows")
            manifest[name] = entry
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
