"""Builds libanu_pdhg.so in-tree with nvcc for sm_100a.

    python -m anukulan_b200.build [--force] [-v]

Objects go to anukulan_b200/_build/ (git-ignored); the shared library lands
next to this file so it travels with the working tree.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libanu_pdhg.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2",
              "--expt-relaxed-constexpr", "-I" + INCLUDE]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-I" + INCLUDE]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source in csrc/ and links libanu_pdhg.so; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    jobs = []
    objs = []
    for src in cu + cpp:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            if src.endswith(".cu"):
                cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
            else:
                cmd = [nvcc(), "-x", "c++"] + ARCH + NVCC_FLAGS + ["-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, flush=True)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or not os.path.exists(LIB):
        link = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        run(link)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
