"""Builds the engine's shared library in-tree: simulated_annealing_b200/libsa_b200.so.

sm_100a only (B200). The library exports the C ABI declared in
include/sa_b200.h and include/sa_b200_batch.h.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libsa_b200.so")
PLAIN = os.path.join(PKG, "sa_plain_pt")  # plain per-instance PT timing program (links LIB)
CLI = os.path.join(PKG, "sa_anneal")  # the command-line front end (links LIB)

SOURCES = ["sa_host.cpp", "sa_system.cu", "sa_batch.cu", "sa_runners.cu", "sa_noalloc.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-Xcompiler", "-Wall",
]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources() -> list[str]:
    return [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h", ".inc"))]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or not up_to_date():
        # one nvcc per source, in parallel, then one link
        objdir = os.path.join(PKG, "_build")
        os.makedirs(objdir, exist_ok=True)
        procs = []
        objs = []
        for src in sources():
            obj = os.path.join(objdir, os.path.basename(src) + ".o")
            cmd = [nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", "-o", obj, src]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            procs.append((subprocess.Popen(cmd), cmd))
            objs.append(obj)
        for p, cmd in procs:
            if p.wait() != 0:
                raise subprocess.CalledProcessError(p.returncode, cmd)
        cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    headers = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    for exe, name in ((PLAIN, "sa_plain_pt.cpp"), (CLI, "sa_cli.cpp")):
        src = os.path.join(CSRC, name)
        newest = max([os.path.getmtime(src), os.path.getmtime(LIB)] + [os.path.getmtime(h) for h in headers])
        if force or not os.path.exists(exe) or os.path.getmtime(exe) < newest:
            cmd = [nvcc(), "-Wno-deprecated-gpu-targets", "-O2", "-std=c++17", "-I", INCLUDE, "-o", exe, src, "-L",
                   PKG, "-lsa_b200", "-Xlinker", "-rpath,$ORIGIN", "-lcudart"]
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
