"""Builds libfomo_b200.so in-tree for sm_100a.

    python -m fomo_julia_b200.build [--verbose]

nvcc cross-compiles without a GPU.  Each translation unit (the runtime and
the split-launch kernels in fomo_b200.cu, one fused-step kernel per order in
march_m<M>.cu) compiles to an object in parallel; the objects link into
``fomo_julia_b200/_lib/libfomo_b200.so``, where the package loads it from.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libfomo_b200.so")
SOURCES = ["fomo_b200.cu", "march_m1.cu", "march_m2.cu", "march_m3.cu", "march_m4.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _deps() -> list[str]:
    out = [os.path.join(REPO, "include", "fomo_b200.h")]
    for n in os.listdir(CSRC):
        if n.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, n))
    return out


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def _compile(src: str, verbose: bool):
    obj = os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", os.path.join(REPO, "include"), *(["-Xptxas", "-v"] if verbose else []),
           "-c", "-o", obj, os.path.join(CSRC, src)]
    return obj, subprocess.run(cmd, capture_output=True, text=True)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    for src, (obj, r) in zip(SOURCES, results):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed for {src}")
        if verbose:
            sys.stderr.write(r.stdout + r.stderr)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *[o for o, _ in results], "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("linking libfomo_b200.so failed")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
