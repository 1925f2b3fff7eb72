"""Tolerance-driven evaluation (bbkde_eval_tol) against the reference's own
dual-tree KernelDensity::eval(queries, rel_err, abs_err) (KernelDensityImpl.h:
624-737, pruning rule :1071-1095), run from oracle/_ref on identical inputs.

The reference's contract: a query's bounds end within rel_err relative or abs_err
absolute, and its value is their midpoint, so |f_ref - f| <= max(rel_err f,
abs_err) / 2. The culled sum promises the same half-allowance plus its own FP32-
compensated arithmetic error (at most 1e-6 f + 1e-9, the bar of the plain FP32C
sum against FP64 that the direct tests hold). Both are checked against the exact
FP64 oracle with the reference's data-point attributes (its exact adaptive pilot
where alpha >= 0), and against each other.
"""
from __future__ import annotations

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [
    # kind, dim, h, alpha
    (W.GAUSS_PROD2D, 2, (0.05, 0.05), 0.5),
    (W.GAUSS, 2, (0.1, 0.1), -1.0),
    (W.EPAN_PROD2D, 2, (0.3, 0.2), -1.0),
    (W.GAUSS, 1, (0.05, 0.05), -1.0),
]
TOLS = [(1e-6, 1e-8), (1e-3, 1e-6)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"k{c[0]}d{c[1]}a{c[3]}")
@pytest.mark.parametrize("tol", TOLS, ids=lambda t: f"rel{t[0]}abs{t[1]}")
def test_eval_tol_matches_reference_tree(ctx, oracle, reference, case, tol):
    kind, dim, h, alpha = case
    rel, abs_ = tol
    wl = W.config2(n=20_000, m=3_000)
    refs = wl.refs if dim == 2 else wl.refs[:, :1].copy()
    q = wl.queries if dim == 2 else wl.queries[:, :1].copy()
    oq, f_ref, (txy, tw, tm, ta) = reference.tree_eval(kind, dim, h, refs, wl.weights, q, rel,
                                                       abs_, alpha=alpha)
    ctx.upload(bk.REFERENCE, txy, mass=tm, abw=ta, weight=tw)
    ctx.upload(bk.QUERY, oq)
    desc = bk.kernel_desc(kind, dim, h)
    got, st = ctx.eval_tol(desc, rel, abs_)
    exact = oracle.direct(kind, dim, h, txy, tm, oq, abw=ta)
    allow = np.maximum(rel * exact, abs_)
    fp32 = 1e-6 * exact + 1e-9 * abs_
    err = np.abs(got - exact)
    worst = int(np.argmax(err - (0.5 * allow + fp32)))
    assert np.all(err <= 0.5 * allow + fp32), (worst, got[worst], exact[worst])
    # the reference's own result holds its contract too, and the two agree
    assert np.all(np.abs(f_ref - exact) <= 0.5 * allow * (1 + 1e-9) + 1e-15)
    assert np.all(np.abs(got - f_ref) <= allow + fp32)
    assert st.max_bound_ratio <= 0.5


def test_eval_tol_arguments(ctx):
    refs = W.f32(W.SplitMix64(3).normal(2000).reshape(1000, 2))
    ctx.upload(bk.REFERENCE, refs, mass=np.full(1000, 1e-3))
    ctx.upload(bk.QUERY, refs[:100])
    desc = bk.kernel_desc(W.GAUSS, 2, (0.2, 0.2))
    for rel, abs_ in ((-1e-3, 0.0), (1.0, 0.0), (1e-6, -1.0), (1e-6, float("inf"))):
        with pytest.raises(bk.InvalidArgument):
            ctx.eval_tol(desc, rel, abs_)
    exact = ctx.eval_all(desc)
    got, _ = ctx.eval_tol(desc, 0.0, 0.0)   # no tolerance: every tile that does not flush
    np.testing.assert_allclose(got, exact, rtol=1e-6)
    with pytest.raises(bk.BBKDEError) as e:
        ctx.eval_tol(bk.kernel_desc(W.EPAN_PROD_CONV2D, 2, (0.2, 0.2)), 1e-6, 1e-8)
    assert e.value.status == bk.UNSUPPORTED
