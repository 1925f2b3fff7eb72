"""Generate the golden vectors under tests/golden/ from the reference's own code.

    python tests/golden/make_golden.py

Runs oracle/_ref/libkde_ref.so -- bbrcit_kde's KernelDensity<> compiled from its
headers by oracle/Makefile -- on seeded inputs from bbrcit_kde_b200.workloads,
and stores inputs' checksums and the reference's outputs as .npz fixtures. The
inputs themselves are regenerated from the seeds at test time.

Every case calls the reference through its public API:
  * direct_eval (KernelDensityImpl.h:1157-1173) at queries,
  * adapt_density (KernelDensityImpl.h:291-359) with rel = abs = 0, which makes
    its dual-tree self-evaluation exact up to FP64 rounding, then direct_eval,
  * likelihood_cross_validate / lsq_convolution_cross_validate (rel = abs = 0).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from bbrcit_kde_b200 import workloads as W  # noqa: E402
from oracle.pyoracle import Reference, build  # noqa: E402


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    return h.hexdigest()


def cases():
    """(name, generator) pairs; each generator returns a dict of inputs."""
    def plain(kind, dim, h, n=2000, steps=40):
        wl = W.config1(n=n, steps=steps)
        refs, q = wl.refs, wl.queries
        if dim == 1:
            refs, q = refs[:, :1].copy(), q[:, :1].copy()
        return dict(kind=kind, dim=dim, h=np.array(h, float), refs=refs,
                    w=np.ones(len(refs)), queries=q, alpha=-1.0)

    def adaptive(kind, h, n=3000, m=800):
        wl = W.config2(n=n, m=m)
        return dict(kind=kind, dim=2, h=np.array(h, float), refs=wl.refs, w=wl.weights,
                    queries=wl.queries, alpha=0.5)

    out = [
        ("cfg1_gauss2d", lambda: plain(W.GAUSS, 2, (0.1, 0.1), n=10_000, steps=100)),
        ("epan2d", lambda: plain(W.EPAN, 2, (0.3, 0.3))),
        ("gaussprod2d", lambda: plain(W.GAUSS_PROD2D, 2, (0.08, 0.15))),
        ("epanprod2d", lambda: plain(W.EPAN_PROD2D, 2, (0.3, 0.2))),
        ("gaussprodconv2d", lambda: plain(W.GAUSS_PROD_CONV2D, 2, (0.08, 0.15))),
        ("epanprodconv2d", lambda: plain(W.EPAN_PROD_CONV2D, 2, (0.3, 0.2))),
        ("gauss1d", lambda: plain(W.GAUSS, 1, (0.02, 0.02))),
        ("epan1d", lambda: plain(W.EPAN, 1, (0.1, 0.1))),
        ("gaussconv1d", lambda: plain(W.GAUSS_CONV1D, 1, (0.05, 0.05))),
        ("epanconv1d", lambda: plain(W.EPAN_CONV1D, 1, (0.1, 0.1))),
        ("cfg2_adaptive_gaussprod2d", lambda: adaptive(W.GAUSS_PROD2D, (0.05, 0.05))),
        ("adaptive_gauss2d", lambda: adaptive(W.GAUSS, (0.1, 0.1))),
    ]
    return out


CV_CASES = [
    # (name, kind, dim, h): LOO likelihood + LSQ-conv on the config-2 style set
    ("cv_gaussprod2d", W.GAUSS_PROD2D, 2, (0.1, 0.15)),
    ("cv_epanprod2d", W.EPAN_PROD2D, 2, (0.4, 0.3)),
    ("cv_gauss1d", W.GAUSS, 1, (0.1, 0.1)),
    ("cv_epan1d", W.EPAN, 1, (0.4, 0.4)),
]


NUMINT_CASES = [
    # (name, kind, h, alpha, grid=(steps_x, steps_y, x0, x1, y0, y1)) on the
    # config-2 style set of 3000 points: lsq_numint_cross_validate
    ("numint_gaussprod2d", W.GAUSS_PROD2D, (0.1, 0.15), -1.0, (64, 48, -3.0, 3.0, -2.5, 2.5)),
    ("numint_epanprod2d", W.EPAN_PROD2D, (0.4, 0.3), -1.0, (64, 48, -3.0, 3.0, -2.5, 2.5)),
    ("numint_gauss2d", W.GAUSS, (0.12, 0.12), -1.0, (80, 80, -3.0, 3.0, -3.0, 3.0)),
    ("numint_epan2d", W.EPAN, (0.3, 0.3), -1.0, (80, 80, -3.0, 3.0, -3.0, 3.0)),
    ("numint_adaptive_gaussprod2d", W.GAUSS_PROD2D, (0.1, 0.15), 0.5,
     (64, 48, -3.0, 3.0, -2.5, 2.5)),
]


def main() -> int:
    build()
    ref = Reference()
    for name, gen in cases():
        d = gen()
        vals, (txy, tw, tm, ta) = ref.eval(d["kind"], d["dim"], d["h"], d["refs"], d["w"],
                                           d["queries"], alpha=d["alpha"])
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"),
            kind=d["kind"], dim=d["dim"], h=d["h"], alpha=d["alpha"],
            n=len(d["refs"]), m=len(d["queries"]),
            input_digest=digest(d["refs"], d["w"], d["queries"]),
            values=vals, tree_xy=txy, tree_w=tw, tree_mass=tm, tree_abw=ta,
            normalization=ref.normalization(d["kind"], d["dim"], d["h"]))
        print(name, len(d["refs"]), len(d["queries"]))
    wl = W.config2(n=3000, m=1)
    for name, kind, dim, h in CV_CASES:
        refs = wl.refs if dim == 2 else wl.refs[:, :1].copy()
        lik = ref.likelihood_cv(kind, dim, h, refs, wl.weights)
        lsq = ref.lsq_conv_cv(kind, dim, h, refs, wl.weights)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), kind=kind, dim=dim,
                            h=np.array(h, float), n=len(refs),
                            input_digest=digest(refs, wl.weights), likelihood=lik, lsq=lsq)
        print(name, lik, lsq)
    for name, kind, h, alpha, grid in NUMINT_CASES:
        cv = ref.lsq_numint_cv(kind, h, wl.refs, wl.weights, grid, alpha=alpha)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), kind=kind, dim=2,
                            h=np.array(h, float), alpha=alpha, grid=np.array(grid, float),
                            n=len(wl.refs), input_digest=digest(wl.refs, wl.weights), cv=cv)
        print(name, cv)
    return 0


if __name__ == "__main__":
    sys.exit(main())
