"""Build libactfem_gpu.so in-tree for sm_100a with nvcc (no JIT cache, no torch extension).

Usage: python -m actfemtide_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libactfem_gpu.so")
OBJ_DIR = os.path.join(HERE, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]
# Files whose arithmetic must round like the serial reference (no FMA contraction).
NOFMA = {"afem_assemble.cu", "afem_sites.cu", "afem_adjoint.cu", "afem_mt.cu"}
SOURCES = ["afem_capi.cu", "afem_mesh.cu", "afem_assemble.cu", "afem_solver.cu", "afem_sites.cu", "afem_mpnn.cu",
           "afem_adjoint.cu", "afem_hybrid.cu", "afem_mt.cu", "afem_io.cpp"]
HEADERS = ["afem_internal.h", "afem_hybrid.h", os.path.join("..", "..", "include", "afem.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    objs, procs = [], []
    for src in SOURCES:
        sp = os.path.join(CSRC, src)
        obj = os.path.join(OBJ_DIR, src + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [sp] + hdrs + [__file__]):
            continue
        cmd = [NVCC] + ARCH + COMMON + ["-c", sp, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
            if src in NOFMA:
                cmd += ["-fmad=false"]
        else:
            cmd += ["-x", "cu"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if verbose and out:
            print(f"--- {src}\n{out}")
        if p.returncode != 0:
            failed.append((src, out))
    if failed:
        msg = "\n".join(f"{s}:\n{o}" for s, o in failed)
        raise RuntimeError(f"nvcc failed:\n{msg}")
    if force or procs or _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
