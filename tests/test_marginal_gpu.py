"""Marginal densities (MarginalDensityAssociator.h:22-128) through the C++ drop-in
(tests/cpp/test_marginal.cc), against the reference's own marginal_density +
direct_eval (oracle/_ref) on identical seeded inputs.

The x (y) marginal of a 2-D product-kernel density is the 1-D density of the x (y)
coordinates with the same weights, the same bandwidth factors, mass = weight /
abw, and the 1-D kernel of the same family with that axis' bandwidth; the drop-in
evaluates it with the device's 1-D pair sums. Bandwidths are exact in FP32, so the
float and double kernels see the same numbers.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from bbrcit_kde_b200.parity import error_stats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_marginal.cc")
BUILD = os.path.join(ROOT, "tests", "cpp", "_build")
EXE = os.path.join(BUILD, "test_marginal")


def compile_marginal() -> str:
    bk.load_library()
    os.makedirs(BUILD, exist_ok=True)
    libdir = os.path.dirname(bk.LIB_PATH)
    subprocess.run(["g++", "-std=c++11", "-O2", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include", "bbkde"),
                    "-I", os.path.join(ROOT, "include"), SRC, "-o", EXE, "-L", libdir,
                    "-lbbkde", "-Wl,-rpath," + libdir], check=True, capture_output=True)
    return EXE


def test_marginal_program_compiles_with_gxx_cxx11():
    assert os.path.exists(compile_marginal())


def _run(exe, tmp_path, kind, fp32, h, alpha, refs, w, q):
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        np.array([len(refs), len(q), kind, int(fp32)], dtype=np.int64).tofile(f)
        np.array([h[0], h[1], alpha], dtype=np.float64).tofile(f)
        np.column_stack([refs, w]).astype(np.float64).tofile(f)
        np.asarray(q, dtype=np.float64).tofile(f)
    r = subprocess.run([exe, str(src), str(dst)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = np.fromfile(dst, dtype=np.uint8)
    m = len(q)
    vals = raw[: 16 * m].view(np.float64)
    fx, fy = vals[:m], vals[m:]
    off = 16 * m
    pts = []
    for _ in range(2):
        k = int(raw[off: off + 8].view(np.int64)[0])
        off += 8
        pts.append(raw[off: off + 32 * k].view(np.float64).reshape(k, 4))
        off += 32 * k
    return fx, fy, pts


@pytest.mark.gpu
@pytest.mark.parametrize("kind", [W.GAUSS_PROD2D, W.EPAN_PROD2D])
@pytest.mark.parametrize("fp32", [True, False])
@pytest.mark.parametrize("alpha", [-1.0, 0.5])
def test_marginals_match_reference(reference, tmp_path, kind, fp32, alpha):
    exe = compile_marginal()
    wl = W.config2(n=4000, m=1)
    h = (0.0625, 0.09375) if kind == W.GAUSS_PROD2D else (0.25, 0.1875)
    q = W.f32(np.linspace(-3.5, 3.5, 1501))   # float-representable, as the device sees them
    fx, fy, (px, py) = _run(exe, tmp_path, kind, fp32, h, alpha, wl.refs, wl.weights, q)
    for dim_idx, got, pts in ((0, fx, px), (1, fy, py)):
        want, (tx, tw, tm, ta) = reference.marginal_direct(kind, h, wl.refs, wl.weights,
                                                           dim_idx, q, alpha=alpha)
        if fp32:
            s = error_stats(got, want, 1e-6, 1e-8)
            assert s["pass_rate"] == 1.0, (dim_idx, s)
        else:
            np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-15)
        # the marginal's points: same coordinates (duplicates merged alike),
        # weights, and mass = weight / abw
        oa = np.lexsort((pts[:, 1], pts[:, 0]))
        ob = np.lexsort((tw, tx))
        np.testing.assert_array_equal(pts[oa, 0], tx[ob])
        np.testing.assert_allclose(pts[oa, 1], tw[ob], rtol=1e-12)
        rtol = 1e-6 if fp32 else 1e-10
        np.testing.assert_allclose(pts[oa, 3], ta[ob], rtol=rtol)
        np.testing.assert_allclose(pts[oa, 2], tm[ob], rtol=2 * rtol)
        np.testing.assert_allclose(pts[:, 2], pts[:, 1] / pts[:, 3], rtol=1e-14)
