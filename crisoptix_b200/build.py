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
SOURCES = ["api.cu", "passes.cu", "search.cu", "reuse_passes.cu", "wavefront.cu", "bvh_build.cpp", "adjoint.cu", "restir_adjoint.cu", "tonemap.cu",
           "context.cpp", "selftest.cu", "radix_sort.cu",
           "bvh_device.cu"]


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


def _flags() -> list:
    return [
        "-ccbin", host_cxx(), "-std=c++17", "-O3", "-lineinfo",
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
        "-I", os.path.join(ROOT, "include"), "-I", CSRC,
    ]


def build(force: bool = False, verbose: bool = False, out: str = OUT, defines=()) -> str:
    """Compile every source to an object in parallel, then link the shared
    library.  Objects go to a build folder beside the sources.  `defines`
    (NAME=VALUE strings) select compile-time variants, built into `out`."""
    if out == OUT and not defines and not force and not needs_build():
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    tag = "_".join(d.replace("=", "") for d in defines)
    objdir = os.path.join(HERE, "_build" + ("_" + tag if tag else ""))
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()

    def compile_one(src: str):
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc] + _flags() + [f"-D{d}" for d in defines] + [
            "-Xptxas", "-v" if verbose else "-O3", "-c", os.path.join(CSRC, src), "-o", obj]
        return subprocess.run(cmd, capture_output=True, text=True), obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    failed = False
    for r, _ in results:
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            failed = True
        elif verbose:
            sys.stderr.write(r.stderr)
    if failed:
        raise RuntimeError("nvcc failed")
    link = [nvcc, "-ccbin", host_cxx(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
            "-o", out + ".tmp"] + [o for _, o in results]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
