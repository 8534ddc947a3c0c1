"""Test infrastructure: compiles the reference's query libraries for the benchmark workloads.

For each workload in WORKLOADS and each reference flavor (hyper, vectorwise), runs the
reference's own code generator through ref_gen (oracle/ref/ref_gen.cpp) and stores
oracle/_ref/<isa>/q_<name>_<flavor>.so.  Generated code depends only on the plan and the
columns' declared min/max, so the libraries run on any table size of the same spec shape.
Needs the reference tree (build host only); the results travel with the repository.

    python oracle/ref/build_queries.py [--isa avx512|avx2]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("VOILA_REFERENCE", "/root/reference")

WORKLOADS = {
    "sel_aggr": "sel_aggr:rows=6000000,seed=1",
    "join_aggr": "join_aggr:build=1500000,probe=6000000,sel=0.2,seed=2",
    "groupby": "groupby:rows=6000000,keys=1500000,zipf=1.25,seed=3",
    "star": "star:rows=60000000,seed=4",
}


def build(isa="avx512", flavors=("hyper", "vectorwise")):
    rdir = os.path.join(REPO, "oracle", "_ref", isa)
    march = "-march=skylake-avx512" if isa == "avx512" else "-march=haswell"
    cxx = (f"g++ {march} -mtune=generic -O3 -g0 -std=c++17 -include cstdint -DIS_RELEASE -w "
           f"-I{HERE}/shim -I{rdir}/gen -I{REF} -I{REF}/libs -I{REF}/db-engine-paradigms/include")
    out = []
    for name, spec in WORKLOADS.items():
        for fl in flavors:
            lib = os.path.join(rdir, f"q_{name}_{fl}.so")
            if os.path.exists(lib) and os.path.getmtime(lib) > os.path.getmtime(os.path.join(rdir, "ref_gen")):
                out.append(lib)
                continue
            r = subprocess.run([os.path.join(rdir, "ref_gen"), "--workload", spec, "--flavor", fl, "--out", lib,
                                "--cxx", cxx], capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"ref_gen failed for {name}/{fl}: {r.stderr[-2000:]}")
            out.append(lib)
    return out


if __name__ == "__main__":
    isa = sys.argv[sys.argv.index("--isa") + 1] if "--isa" in sys.argv else "avx512"
    for lib in build(isa):
        print(lib)
