"""Test infrastructure: compiles the reference's query libraries for the benchmark workloads.

For each workload in WORKLOADS and each reference flavor (hyper, vectorwise), runs the
reference's own code generator through ref_gen (oracle/ref/ref_gen.cpp) and stores
oracle/_ref/<isa>/q_<name>_<flavor>.so.  Generated code depends only on the plan and the
columns' declared min/max, so the libraries run on any table size of the same spec shape.

It also builds the CUDA flavor's generated libraries (ref_gen --flavor cuda: the plan through
the reference's relalg tree into the glue of cuda_glue.inc over libvoila_cuda.so) for the
same workloads and for every golden case, q_<name>_cuda.so and q_golden_<case>_cuda.so, which
ref_run drives through the reference's voila_query_* ABI in the GPU tests.
Needs the reference tree (build host only); the results travel with the repository.

    python oracle/ref/build_queries.py [--isa avx512|avx2]
"""
import json
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


def _cuda_libs():
    """(library name, workload spec, plan or None) of the CUDA-flavor glue libraries."""
    out = [(f"q_{name}_cuda", spec, None) for name, spec in WORKLOADS.items()]
    with open(os.path.join(REPO, "tests", "golden", "manifest.json")) as f:
        for case, entry in sorted(json.load(f).items()):
            out.append((f"q_golden_{case}_cuda", entry["spec"], entry["plan"]))
    return out


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
    glue_deps = [os.path.join(rdir, "ref_gen"), os.path.join(HERE, "cuda_glue.inc"),
                 os.path.join(REPO, "include", "voila_cuda.h")]
    stamp = max(os.path.getmtime(d) for d in glue_deps)
    link = ("-L" + os.path.join(REPO, "vldb_voila_b200") + " -lvoila_cuda"
            " -Wl,-rpath,'$ORIGIN/../../../vldb_voila_b200'")
    for name, spec, plan in _cuda_libs():
        lib = os.path.join(rdir, name + ".so")
        if os.path.exists(lib) and os.path.getmtime(lib) > stamp:
            out.append(lib)
            continue
        cmd = [os.path.join(rdir, "ref_gen"), "--workload", spec, "--flavor", "cuda", "--out", lib,
               "--cxx", cxx + f" -I{HERE} -I{REPO}/include", "--link", link]
        if plan:
            cmd += ["--plan", plan]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"ref_gen failed for {name}: {r.stderr[-2000:]}")
        out.append(lib)
    return out


if __name__ == "__main__":
    isa = sys.argv[sys.argv.index("--isa") + 1] if "--isa" in sys.argv else "avx512"
    for lib in build(isa):
        print(lib)
