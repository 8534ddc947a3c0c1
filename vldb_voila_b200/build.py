"""Builds libvoila_cuda.so in-tree: the CUDA flavor's host runtime (C++), its ahead-of-time
sm_100a kernels (nvcc) and the embedded device header that NVRTC compiles pipelines against.

    python -m vldb_voila_b200.build            # incremental
    python -m vldb_voila_b200.build --force    # rebuild everything
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
REPO = os.path.dirname(HERE)
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
LIB = os.path.join(HERE, "libvoila_cuda.so")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xptxas", "-v"]
CXX_FLAGS = ["-O2", "-g", "-fPIC", "-std=c++17", "-Wall", "-Wno-unused-function", "-ffp-contract=off"]

CPP_SOURCES = ["engine.cpp", "plan.cpp", "codegen.cpp", "jit.cpp", "batch.cpp", "import.cpp"]
CU_SOURCES = ["datagen.cu", "mlp.cu", "noalloc.cu", "floor.cu"]
HEADERS = ["datagen.h", "engine_internal.hpp", "sexpr.hpp", "workloads.hpp", "device/voila_device.cuh"]


def _run(cmd, log=None):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.append(r.stderr)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + cmd[0] + " " + cmd[-1])
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _embed_header():
    src = os.path.join(CSRC, "device", "voila_device.cuh")
    out = os.path.join(BUILD, "device_header.inc")
    if not _stale(out, [src, __file__]):
        return out
    text = open(src).read()
    delim = "VDHDR"
    assert (")" + delim + '"') not in text
    with open(out, "w") as f:
        f.write("/* generated from csrc/device/voila_device.cuh by build.py */\n")
        f.write('static const char* kDeviceHeader = R"' + delim + "(" + text + ")" + delim + '";\n')
    return out


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    _embed_header()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(REPO, "include", "voila_cuda.h")]
    objs = []
    ptxas_log = []
    for cu in CU_SOURCES:
        src = os.path.join(CSRC, cu)
        obj = os.path.join(BUILD, cu + ".o")
        if force or _stale(obj, [src] + hdrs):
            _run([os.path.join(CUDA, "bin", "nvcc")] + NVCC_FLAGS + ["-I", CSRC, "-c", src, "-o", obj], ptxas_log)
        objs.append(obj)
    for cpp in CPP_SOURCES:
        src = os.path.join(CSRC, cpp)
        obj = os.path.join(BUILD, cpp + ".o")
        deps = [src] + hdrs + [os.path.join(BUILD, "device_header.inc")]
        if force or _stale(obj, deps):
            _run(["g++"] + CXX_FLAGS + ["-I", CSRC, "-I", BUILD, "-I", os.path.join(CUDA, "include"),
                                        "-c", src, "-o", obj])
        objs.append(obj)
    if force or _stale(LIB, objs):
        _run(["g++", "-shared", "-o", LIB] + objs +
             ["-L" + os.path.join(CUDA, "lib64"), "-lcudart_static", "-lnvrtc", "-lpthread", "-ldl", "-lrt",
              "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-Wl,--no-undefined"])
    if verbose:
        for l in ptxas_log:
            if l.strip():
                print(l)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
