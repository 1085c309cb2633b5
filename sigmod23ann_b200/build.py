"""Builds libknng.so in-tree: every .cu under csrc/ compiled for sm_100a.

    python -m sigmod23ann_b200.build [--verbose-ptxas]

Objects go to sigmod23ann_b200/_build/ and the shared library to
sigmod23ann_b200/libknng.so (both git-ignored; the library travels with the
repository to a GPU host).  Objects are rebuilt when their source or any
header changed.
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libknng.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
         "-ccbin", "/usr/bin/g++", "-I", CSRC, "-I", INCLUDE]


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = _headers()
    objects = []
    for src in sources:
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objects.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objects):
        subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objects, "-ccbin", "/usr/bin/g++"], check=True)
    # Command-line tools: the reference's program shape (contest file in,
    # output.bin out) and its grader.
    for name, link in (("knng_build", True), ("knng_grade", False)):
        src = os.path.join(HERE, "cli", name + ".cpp")
        exe = os.path.join(HERE, "cli", name)
        if force or _stale(exe, [src, LIB] if link else [src]):
            cmd = ["/usr/bin/g++", "-O2", "-std=c++17", "-I", INCLUDE, src, "-o", exe]
            if link:
                cmd += [f"-L{HERE}", "-lknng", f"-Wl,-rpath,{HERE}"]
            subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.verbose_ptxas, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
