"""Batched cross-validation (bbkde_cv_batch) against the per-bandwidth path and
the reference's own CV values."""
from __future__ import annotations

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from tests.helpers import load_golden

pytestmark = pytest.mark.gpu


def _per_bandwidth(ctx, kind, datasets, hx, hy):
    """The reference's loop: one likelihood / LSQ CV per bandwidth pair (FP64)."""
    lik = np.empty((len(datasets), len(hx), len(hy)))
    lsq = np.empty_like(lik)
    for s, (xy, w) in enumerate(datasets):
        wn = (np.ones(len(xy)) if w is None else w) / (len(xy) if w is None else w.sum())
        ctx.upload(bk.REFERENCE, xy, mass=wn, weight=wn)
        for a, x in enumerate(hx):
            for b, y in enumerate(hy):
                d = bk.kernel_desc(kind, 2, (x, y))
                lik[s, a, b] = ctx.likelihood_cv(d, bk.FP64)
                lsq[s, a, b] = ctx.lsq_conv_cv(d, bk.FP64)
    return lik, lsq


def _close(got, want, rtol):
    both_inf = np.isinf(got) & np.isinf(want) & (np.sign(got) == np.sign(want))
    ok = both_inf | np.isclose(got, want, rtol=rtol, atol=0)
    assert ok.all(), (got[~ok][:5], want[~ok][:5])


def test_cv_batch_matches_per_bandwidth_loop(ctx):
    sets = W.config3_datasets(n_sets=3, sizes=[1500, 2600, 700])
    rng = W.SplitMix64(42)
    datasets = [(sets[0], None), (sets[1], rng.uniform(2600, 0.5, 1.5)), (sets[2], None)]
    grid = W.config3_bandwidths()
    hx, hy = grid[::6], grid[3::7]          # 11 x 9, spanning [0.01, 1]
    lik, lsq = ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, datasets, hx, hy)
    want_lik, want_lsq = _per_bandwidth(ctx, bk.EPANECHNIKOV_PRODUCT_2D, datasets, hx, hy)
    _close(lik, want_lik, 1e-9)
    _close(lsq, want_lsq, 1e-9)
    assert np.isfinite(lsq).all()


def test_cv_batch_full_grid_sampled(ctx):
    """All 64 x 64 bandwidths for two larger datasets in one call, checked on a
    sample of grid points against the per-bandwidth path."""
    sets = W.config3_datasets(n_sets=2, sizes=[20000, 6000])
    datasets = [(s, None) for s in sets]
    h = W.config3_bandwidths()
    lik, lsq = ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, datasets, h, h)
    assert lik.shape == (2, 64, 64)
    picks = [(0, 0), (5, 60), (31, 32), (63, 63), (40, 7), (63, 0), (20, 50)]
    for s, (xy, _) in enumerate(datasets):
        wn = np.full(len(xy), 1.0 / len(xy))
        ctx.upload(bk.REFERENCE, xy, mass=wn, weight=wn)
        for a, b in picks:
            d = bk.kernel_desc(bk.EPANECHNIKOV_PRODUCT_2D, 2, (h[a], h[b]))
            _close(np.array([lik[s, a, b]]), np.array([ctx.likelihood_cv(d, bk.FP64)]), 1e-9)
            _close(np.array([lsq[s, a, b]]), np.array([ctx.lsq_conv_cv(d, bk.FP64)]), 1e-9)
    # the graph is replayed for a second call of the same shape
    lik2, lsq2 = ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, datasets, h, h)
    _close(lik2, lik, 1e-12)
    _close(lsq2, lsq, 1e-12)


def test_cv_batch_matches_reference_golden(ctx):
    """The reference's own likelihood / LSQ-conv CV (tests/golden/cv_epanprod2d)."""
    g = load_golden("cv_epanprod2d")
    wl = W.config2(n=3000, m=1)
    h = tuple(g["h"])
    lik, lsq = ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, [(wl.refs, wl.weights)], [h[0]],
                            [h[1]])
    assert lik[0, 0, 0] == pytest.approx(float(g["likelihood"]), rel=1e-10)
    assert lsq[0, 0, 0] == pytest.approx(float(g["lsq"]), rel=1e-10)


def test_cv_batch_gaussian_loop_and_errors(ctx):
    sets = W.config3_datasets(n_sets=1, sizes=[900])
    datasets = [(sets[0], None)]
    hx, hy = [0.05, 0.2], [0.1, 0.3, 0.6]
    lik, lsq = ctx.cv_batch(bk.GAUSSIAN_PRODUCT_2D, datasets, hx, hy)
    want_lik, want_lsq = _per_bandwidth(ctx, bk.GAUSSIAN_PRODUCT_2D, datasets, hx, hy)
    _close(lik, want_lik, 1e-12)
    _close(lsq, want_lsq, 1e-12)
    with pytest.raises(bk.InvalidArgument):
        ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, datasets, [0.2, 0.1], hy)   # not increasing
    with pytest.raises(bk.InvalidArgument):
        ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, datasets, np.linspace(0.01, 1, 65), hy)
    with pytest.raises(bk.BBKDEError):
        ctx.cv_batch(bk.GAUSSIAN, datasets, hx, hy)


def test_cv_batch_plans_and_autotuner(ctx):
    """Every work-item plan gives the same scores to FP64 rounding (the likelihood
    sums are grouped per work item; the LSQ moments are exact integers, but the
    score subtracts twice the grouped leave-one-out sum); without a forced plan the first calls of
    a problem class run each plan once, then the fastest is kept; the launch
    statistics count the in-support pairs."""
    sets = W.config3_datasets(n_sets=2, sizes=[9000, 3000])
    datasets = [(s, None) for s in sets]
    h = W.config3_bandwidths()[::4]
    res = []
    for plan in range(3):
        ctx.set_cv_plan(plan)
        res.append(ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, datasets, h, h))
        lik_pairs, conv_pairs, used, n_plans = ctx.cv_batch_info()
        assert used == plan and n_plans == 3
        assert 0 < lik_pairs <= 9000 ** 2 + 3000 ** 2
        assert 0 < conv_pairs <= (9000 ** 2 + 3000 ** 2) // 2
    for lik, lsq in res[1:]:
        _close(lik, res[0][0], 1e-12)
        _close(lsq, res[0][1], 1e-12)
    with pytest.raises(bk.InvalidArgument):
        ctx.set_cv_plan(3)
    ctx.set_cv_plan(-1)
    sets2 = W.config3_datasets(n_sets=3, sizes=[5000, 4000, 3000])   # a new problem class
    ds2 = [(s, None) for s in sets2]
    used = []
    for _ in range(5):
        ctx.cv_batch(bk.EPANECHNIKOV_PRODUCT_2D, ds2, h, h)
        used.append(ctx.cv_batch_info()[2])
    assert sorted(used[:3]) == [0, 1, 2]
    assert used[3] == used[4]
