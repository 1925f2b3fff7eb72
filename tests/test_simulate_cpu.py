"""KernelDensity::simulate through the C++ drop-in (KernelDensityImpl.h:99-138):
a data point drawn with probability equal to its weight, plus a draw from the
kernel scaled by the point's bandwidth factor (abw). Host code only (no device).

Each kernel's samples are compared with the density they should follow: the
marginal CDF of every coordinate, sum_i w_i K_cdf((t - x_i) / (h_axis abw_i)),
by a Kolmogorov-Smirnov distance, and in 2-D the mixed moment E[xy] with its
standard error (the kernels are uncorrelated, so E[xy] = sum_i w_i x_i y_i).
Sample size 2,000,000: a KS distance above 0.002 has probability below 1e-6 under
the hypothesis, while drawing points uniformly instead of by weight, or dropping
the bandwidth factor, moves it to about 0.005; the seeds are fixed, so the
outcome is deterministic.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest
from scipy.special import ndtr

import bbrcit_kde_b200 as bk

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_simulate.cc")
BUILD = os.path.join(ROOT, "tests", "cpp", "_build")
EXE = os.path.join(BUILD, "test_simulate")
N = 2_000_000


def epan1_cdf(u):
    u = np.clip(u, -1.0, 1.0)
    return 0.5 + 0.75 * (u - u ** 3 / 3.0)


def epan2_axis_cdf(u):
    # marginal of (2/pi)(1 - r^2) on the unit disk: (8 / 3pi)(1 - x^2)^(3/2)
    u = np.clip(u, -1.0, 1.0)
    s = np.sqrt(1.0 - u * u)
    prim = (u * (5.0 - 2.0 * u * u) * s + 3.0 * np.arcsin(u)) / 8.0
    return 0.5 + 8.0 / (3.0 * np.pi) * prim


# kernel -> (dim, per-axis bandwidths, per-axis unit CDF, per-axis unit variance)
KERNELS = {
    "gprod": (2, (0.1, 0.2), ndtr, 1.0),
    "gauss2": (2, (0.15, 0.15), ndtr, 1.0),
    "eprod": (2, (0.3, 0.2), epan1_cdf, 0.2),
    "epan2": (2, (0.25, 0.25), epan2_axis_cdf, 1.0 / 6.0),
    "epan1": (1, (0.2,), epan1_cdf, 0.2),
    "gauss1": (1, (0.1,), ndtr, 1.0),
}


@pytest.fixture(scope="module")
def exe():
    bk.load_library()
    os.makedirs(BUILD, exist_ok=True)
    libdir = os.path.dirname(bk.LIB_PATH)
    subprocess.run(["g++", "-std=c++11", "-O2", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include", "bbkde"),
                    "-I", os.path.join(ROOT, "include"), SRC, "-o", EXE, "-L", libdir,
                    "-lbbkde", "-Wl,-rpath," + libdir], check=True, capture_output=True)
    return EXE


def _draw(exe, kernel, tmp_path):
    path = str(tmp_path / f"{kernel}.bin")
    subprocess.run([exe, kernel, str(N), path], check=True, timeout=120)
    raw = np.fromfile(path, dtype=np.int64, count=2)
    n_pts, dim = int(raw[0]), int(raw[1])
    vals = np.fromfile(path, dtype=np.float64, offset=16)
    pts = vals[: n_pts * (dim + 2)].reshape(n_pts, dim + 2)
    samples = vals[n_pts * (dim + 2):].reshape(-1, dim)
    return pts[:, :dim], pts[:, dim], pts[:, dim + 1], samples


@pytest.mark.parametrize("kernel", sorted(KERNELS))
def test_simulate_follows_the_density(exe, kernel, tmp_path):
    dim, h, cdf, var_k = KERNELS[kernel]
    x, w, abw, s = _draw(exe, kernel, tmp_path)
    assert s.shape == (N, dim) and np.all(np.isfinite(s))
    assert abs(w.sum() - 1.0) < 1e-12          # the constructor normalised the weights
    for ax in range(dim):
        t = np.quantile(s[:, ax], np.linspace(0.0005, 0.9995, 2000))
        model = (w[None, :] * cdf((t[:, None] - x[None, :, ax]) / (h[ax] * abw[None, :]))).sum(1)
        emp = np.searchsorted(np.sort(s[:, ax]), t, side="right") / N
        ks = np.max(np.abs(emp - model))
        assert ks < 0.002, (kernel, ax, ks)
        # the mean, with its standard error
        mu = float((w * x[:, ax]).sum())
        se = s[:, ax].std() / np.sqrt(N)
        assert abs(s[:, ax].mean() - mu) < 6 * se, (kernel, ax)
        # the variance: spread of the points plus the scaled kernel's variance
        var = float((w * (x[:, ax] - mu) ** 2).sum() + (w * (h[ax] * abw) ** 2).sum() * var_k)
        d2 = (s[:, ax] - mu) ** 2
        assert abs(d2.mean() - var) < 6 * d2.std() / np.sqrt(N), (kernel, ax)
    if dim == 2:
        xy = s[:, 0] * s[:, 1]
        want = float((w * x[:, 0] * x[:, 1]).sum())
        assert abs(xy.mean() - want) < 6 * xy.std() / np.sqrt(N), kernel
