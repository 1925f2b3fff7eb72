"""Test helpers: golden fixtures and parity assertions."""
from __future__ import annotations

import hashlib
import os

import numpy as np

from bbrcit_kde_b200 import workloads as W
from bbrcit_kde_b200.parity import error_stats

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Golden case -> generator of its inputs (mirrors tests/golden/make_golden.py).
PLAIN_CASES = {
    "cfg1_gauss2d": (W.GAUSS, 2, (0.1, 0.1), 10_000, 100),
    "epan2d": (W.EPAN, 2, (0.3, 0.3), 2000, 40),
    "gaussprod2d": (W.GAUSS_PROD2D, 2, (0.08, 0.15), 2000, 40),
    "epanprod2d": (W.EPAN_PROD2D, 2, (0.3, 0.2), 2000, 40),
    "gaussprodconv2d": (W.GAUSS_PROD_CONV2D, 2, (0.08, 0.15), 2000, 40),
    "epanprodconv2d": (W.EPAN_PROD_CONV2D, 2, (0.3, 0.2), 2000, 40),
    "gauss1d": (W.GAUSS, 1, (0.02, 0.02), 2000, 40),
    "epan1d": (W.EPAN, 1, (0.1, 0.1), 2000, 40),
    "gaussconv1d": (W.GAUSS_CONV1D, 1, (0.05, 0.05), 2000, 40),
    "epanconv1d": (W.EPAN_CONV1D, 1, (0.1, 0.1), 2000, 40),
}
ADAPTIVE_CASES = {
    "cfg2_adaptive_gaussprod2d": (W.GAUSS_PROD2D, (0.05, 0.05)),
    "adaptive_gauss2d": (W.GAUSS, (0.1, 0.1)),
}
CV_CASES = {
    "cv_gaussprod2d": (W.GAUSS_PROD2D, 2, (0.1, 0.15)),
    "cv_epanprod2d": (W.EPAN_PROD2D, 2, (0.4, 0.3)),
    "cv_gauss1d": (W.GAUSS, 1, (0.1, 0.1)),
    "cv_epan1d": (W.EPAN, 1, (0.4, 0.4)),
}


NUMINT_CASES = {
    # name -> (kind, h, alpha, grid=(steps_x, steps_y, x0, x1, y0, y1))
    "numint_gaussprod2d": (W.GAUSS_PROD2D, (0.1, 0.15), -1.0, (64, 48, -3.0, 3.0, -2.5, 2.5)),
    "numint_epanprod2d": (W.EPAN_PROD2D, (0.4, 0.3), -1.0, (64, 48, -3.0, 3.0, -2.5, 2.5)),
    "numint_gauss2d": (W.GAUSS, (0.12, 0.12), -1.0, (80, 80, -3.0, 3.0, -3.0, 3.0)),
    "numint_epan2d": (W.EPAN, (0.3, 0.3), -1.0, (80, 80, -3.0, 3.0, -3.0, 3.0)),
    "numint_adaptive_gaussprod2d": (W.GAUSS_PROD2D, (0.1, 0.15), 0.5,
                                    (64, 48, -3.0, 3.0, -2.5, 2.5)),
}


def numint_inputs(name):
    kind, h, alpha, grid = NUMINT_CASES[name]
    wl = W.config2(n=3000, m=1)
    return kind, h, alpha, grid, wl.refs, wl.weights


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def plain_inputs(name):
    kind, dim, h, n, steps = PLAIN_CASES[name]
    wl = W.config1(n=n, steps=steps)
    refs, q = wl.refs, wl.queries
    if dim == 1:
        refs, q = refs[:, :1].copy(), q[:, :1].copy()
    return kind, dim, h, refs, np.ones(len(refs)), q


def adaptive_inputs(name):
    kind, h = ADAPTIVE_CASES[name]
    wl = W.config2(n=3000, m=800)
    return kind, 2, h, wl.refs, wl.weights, wl.queries


def cv_inputs(name):
    kind, dim, h = CV_CASES[name]
    wl = W.config2(n=3000, m=1)
    refs = wl.refs if dim == 2 else wl.refs[:, :1].copy()
    return kind, dim, h, refs, wl.weights


def match_by_coords(xy_a, xy_b):
    """Permutations pa, pb with xy_a[pa] == xy_b[pb] (lexicographic order)."""
    xy_a = np.asarray(xy_a).reshape(len(xy_a), -1)
    xy_b = np.asarray(xy_b).reshape(len(xy_b), -1)
    pa = np.lexsort(xy_a.T[::-1])
    pb = np.lexsort(xy_b.T[::-1])
    return pa, pb


def assert_parity(got, ref, rel_err=1e-6, abs_err=1e-8, min_pass=1.0, what=""):
    s = error_stats(got, ref, rel_err, abs_err)
    assert s["pass_rate"] >= min_pass, f"{what}: {s}"
    return s
