"""Builds libsc_gpu.so (the sm_100a kernels and the C ABI of include/sc_gpu.h).

Every translation unit is compiled for sm_100a only, with -fmad=false so that
no f64 a*b+c is contracted into an FMA (the reference's arithmetic never is).
Objects go to _build/, the library next to the Python package (sc_gpu/), so
it travels with the source tree.

Usage: python single-clustering_b200/build.py [--verbose-ptxas] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "sc_gpu", "libsc_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O2", "-I" + INCLUDE, "-I" + CSRC,
]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose_ptxas: bool = False, jobs: int = 8, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "sc_gpu.h"))
    objs = []
    todo = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or verbose_ptxas or not _newer(obj, [src] + headers):
            flags = list(NVCC_FLAGS)
            if verbose_ptxas:
                flags += ["-Xptxas", "-v"]
            todo.append([nvcc(), *flags, "-c", src, "-o", obj])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    failed = False
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for cmd, r in ex.map(run, todo):
            out = (r.stdout or "") + (r.stderr or "")
            if r.returncode != 0:
                failed = True
                sys.stderr.write(f"FAILED: {' '.join(cmd)}\n{out}\n")
            elif verbose_ptxas and out.strip():
                sys.stderr.write(out)
    if failed:
        raise RuntimeError("nvcc failed")
    if todo or not _newer(OUT, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return OUT


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=8)
    a = ap.parse_args()
    print(build(a.verbose_ptxas, a.j, a.force))


if __name__ == "__main__":
    main()
