"""Builds libfomo_b200.so in-tree for sm_100a.

    python -m fomo_julia_b200.build [--verbose]

nvcc cross-compiles without a GPU.  The library is written to
``fomo_julia_b200/_lib/libfomo_b200.so``, where the package loads it from.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libfomo_b200.so")
SOURCES = ["fomo_b200.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2",
         "-shared", "--expt-relaxed-constexpr"]


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


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", os.path.join(REPO, "include"),
           *(["-Xptxas", "-v"] if verbose else []),
           "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES], "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed for libfomo_b200.so")
    if verbose:
        sys.stderr.write(r.stdout + r.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
