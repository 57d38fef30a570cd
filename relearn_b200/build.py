"""Build recipe for librelearn_b200.so (sm_100a, in-tree)."""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "librelearn_b200.so")
SOURCES = ["prims.cu", "octree.cu", "bh_search.cu", "connector.cu", "activity.cu", "capi.cu", "noalloc.cu", "fp32.cu", "serve.cpp"]
HEADERS = ["rl_internal.cuh", "rl_context.cuh", "rl_math.cuh", "bh_eval.cuh"]
INCLUDE = os.path.join(os.path.dirname(HERE), "include", "relearn_b200.h")

# -fmad=false: no multiply-add contraction, so FP64 results match the CPU
# oracle (compiled with -ffp-contract=off) bit for bit.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


HOST = os.path.join(HERE, "host")
BIN = os.path.join(HERE, "bin")
HOST_PROGRAMS = ["relearn_b200_run", "host_selftest"]


def stale() -> bool:
    outs = [LIB] + [os.path.join(BIN, p) for p in HOST_PROGRAMS]
    if not all(os.path.exists(o) for o in outs):
        return True
    t = min(os.path.getmtime(o) for o in outs)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [INCLUDE, __file__]
    deps += [os.path.join(HOST, f) for f in os.listdir(HOST)]
    return any(os.path.getmtime(d) > t for d in deps)


def build_host(verbose: bool = False) -> None:
    """The C++ host programs over the C ABI (C++20, linked to the library in
    this directory through an rpath)."""
    os.makedirs(BIN, exist_ok=True)
    cxx = os.environ.get("CXX", "g++")
    for prog in HOST_PROGRAMS:
        cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-Wextra", "-o", os.path.join(BIN, prog), os.path.join(HOST, prog + ".cpp"), "-L" + HERE,
               "-lrelearn_b200", "-Wl,-rpath,$ORIGIN/.."]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    objs = [os.path.join(CSRC, os.path.splitext(src)[0] + ".o") for src in SOURCES]
    cmds = [[nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj] for src, obj in zip(SOURCES, objs)]
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd), file=sys.stderr)
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as pool:
        for res in pool.map(lambda cmd: subprocess.run(cmd, capture_output=True, text=True), cmds):
            if res.returncode != 0:
                sys.stderr.write(res.stdout + res.stderr)
                raise subprocess.CalledProcessError(res.returncode, res.args)
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-Xcompiler", "-pthread", "-o", LIB, *objs]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    build_host(verbose)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
