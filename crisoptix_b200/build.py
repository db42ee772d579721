"""Build the CUDA library libcrisb.so in-tree for sm_100a.

The device code relies on IEEE float semantics for reproducible results:
no fast-math, no FMA contraction (-fmad=false), IEEE division and square root.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcrisb.so")
SOURCES = ["api.cu", "passes.cu", "search.cu", "reuse_passes.cu", "wavefront.cu", "bvh_build.cpp", "adjoint.cu", "tonemap.cu"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "crisb.h"),
                                                                 os.path.abspath(__file__)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    cmd = [
        nvcc_path(), "-ccbin", host_cxx(), "-std=c++17", "-O3", "-lineinfo",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
        "-Xptxas", "-v" if verbose else "-O3",
        "-shared", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
        "-o", OUT + ".tmp",
    ] + [os.path.join(CSRC, s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
