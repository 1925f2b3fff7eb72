"""Build libbbkde.so (the C-ABI CUDA library) in-tree for sm_100a.

    python -m bbrcit_kde_b200.build            # build if sources changed
    python -m bbrcit_kde_b200.build --force    # rebuild
    python -m bbrcit_kde_b200.build --ptxas-info   # print registers / spills

The library is compiled by nvcc straight from csrc/ with
``-gencode arch=compute_100a,code=sm_100a`` and the CUDA runtime linked
statically, so the resulting .so depends on the driver only.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libbbkde.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + \
        sorted(glob.glob(os.path.join(INCLUDE, "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in deps())


def build(force: bool = False, ptxas_info: bool = False, verbose: bool = False) -> str:
    if not force and not ptxas_info and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "-Xlinker", "--exclude-libs,ALL",
           "-I", INCLUDE, "-o", tmp, *sources()]
    if ptxas_info:
        cmd.insert(1, "-Xptxas=-v")
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


GRID_SEARCH_SRC = os.path.join(PKG, "grid_search", "grid_search.cc")
GRID_SEARCH = os.path.join(LIBDIR, "grid_search")


def build_grid_search(force: bool = False) -> str:
    """The grid_search command-line driver: plain g++ over the C ABI, rpath to lib/."""
    lib = build()
    if (not force and os.path.exists(GRID_SEARCH) and
            os.path.getmtime(GRID_SEARCH) >= max(os.path.getmtime(GRID_SEARCH_SRC),
                                                 os.path.getmtime(lib))):
        return GRID_SEARCH
    cxx = shutil.which("g++") or "g++"
    tmp = GRID_SEARCH + ".tmp"
    subprocess.check_call([cxx, "-std=c++11", "-O2", "-Wall", "-Wextra", "-Werror",
                           GRID_SEARCH_SRC, "-o", tmp, "-L", LIBDIR, "-lbbkde",
                           "-Wl,-rpath,$ORIGIN"])
    os.replace(tmp, GRID_SEARCH)
    return GRID_SEARCH


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, ptxas_info=a.ptxas_info, verbose=a.verbose))
    print(build_grid_search(force=a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
