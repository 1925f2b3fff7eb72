"""The C++ drop-in headers (include/bbkde/) compile with g++ as reference code
does and, on a GPU, reproduce FP64 CPU loops (tests/cpp/test_dropin.cc)."""
from __future__ import annotations

import os
import subprocess

import pytest

import bbrcit_kde_b200 as bk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_dropin.cc")
BUILD = os.path.join(ROOT, "tests", "cpp", "_build")
EXE = os.path.join(BUILD, "test_dropin")


def compile_dropin() -> str:
    bk.load_library()   # builds libbbkde.so if needed
    os.makedirs(BUILD, exist_ok=True)
    libdir = os.path.dirname(bk.LIB_PATH)
    cmd = ["g++", "-std=c++11", "-O2", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include", "bbkde"), "-I", os.path.join(ROOT, "include"),
           SRC, "-o", EXE, "-L", libdir, "-lbbkde", "-Wl,-rpath," + libdir]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return EXE


def test_dropin_compiles_with_gxx_cxx11():
    assert os.path.exists(compile_dropin())


def _has_gpu() -> bool:
    import torch
    return torch.cuda.is_available()


@pytest.mark.skipif(_has_gpu(), reason="a GPU is present")
def test_dropin_without_gpu_fails_loudly():
    exe = compile_dropin()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 2, r.stdout
    assert "no CUDA device" in r.stdout


@pytest.mark.gpu
def test_dropin_matches_cpu_fp64_loops():
    exe = compile_dropin()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ALL PASSED" in r.stdout and "FAILED" not in r.stdout
