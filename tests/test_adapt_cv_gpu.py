"""Parity of the adaptive pilot and the cross-validation sums (through the C ABI)
with the reference's golden vectors and the FP64 oracle."""
from __future__ import annotations

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from tests.helpers import (ADAPTIVE_CASES, CV_CASES, NUMINT_CASES, adaptive_inputs,
                           assert_parity, cv_inputs, load_golden, match_by_coords,
                           numint_inputs)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(ADAPTIVE_CASES))
@pytest.mark.parametrize("precision", [bk.FP32C, bk.FP64])
def test_adapt_density_matches_golden(ctx, oracle, name, precision):
    g = load_golden(name)
    kind, dim, h, refs, w, q = adaptive_inputs(name)
    wn = w / w.sum()
    ctx.upload(bk.REFERENCE, refs, mass=wn, weight=wn)
    ctx.upload(bk.QUERY, q)
    desc = bk.kernel_desc(kind, dim, h)
    abw, mass, pilot, gm = ctx.adapt_density(desc, 0.5, precision)
    pa, pb = match_by_coords(refs, g["tree_xy"].reshape(-1, dim))
    # FP32C: the pilot sums are FP32-compensated (~1e-7), g and the attributes
    # FP64, so abw and mass hold the 1e-6 relative bar of FP32-compensated sums.
    rtol = 1e-10 if precision == bk.FP64 else 1e-6
    np.testing.assert_allclose(abw[pa], g["tree_abw"][pb], rtol=rtol)
    np.testing.assert_allclose(mass[pa], g["tree_mass"][pb], rtol=rtol * 2)
    _, _, _, g_or = oracle.adapt(kind, dim, h, refs, wn, 0.5)
    assert gm == pytest.approx(g_or, rel=rtol)
    # attributes stay on the device: the next evaluation is adaptive
    m_dev, a_dev = ctx.download_attributes()
    np.testing.assert_array_equal(a_dev, abw)
    vals = ctx.eval_all(desc, precision=precision)
    if precision == bk.FP64:
        np.testing.assert_allclose(vals, g["values"], rtol=1e-9)
    else:
        # the reference's own CPU-vs-GPU criterion approximately_equal(1e-6, 1e-8)
        # at every query (pilot and evaluation both FP32-compensated)
        s = assert_parity(vals, g["values"], 1e-6, 1e-8, what=name)
        assert s["max_rel_1e3"] <= 1e-6, s


def test_adapt_alpha_validation_and_reset(ctx):
    refs = W.f32(W.SplitMix64(1).normal(200).reshape(100, 2))
    w = np.full(100, 0.01)
    ctx.upload(bk.REFERENCE, refs, mass=w, weight=w)
    d = bk.kernel_desc(W.GAUSS, 2, (0.3,))
    for alpha in (-0.01, 1.01, float("nan")):
        with pytest.raises(bk.InvalidArgument):
            ctx.adapt_density(d, alpha)
    abw, mass, _, _ = ctx.adapt_density(d, 0.5)
    assert not np.allclose(abw, 1.0)
    abw0, mass0, _, _ = ctx.adapt_density(d, 0.0)   # alpha = 0: unadapted
    np.testing.assert_array_equal(abw0, np.ones(100))
    np.testing.assert_array_equal(mass0, w)
    ctx.adapt_density(d, 0.7)
    ctx.unadapt_density()
    m, a = ctx.download_attributes()
    np.testing.assert_array_equal(a, np.ones(100))
    np.testing.assert_array_equal(m, w)


@pytest.mark.parametrize("name", sorted(CV_CASES))
@pytest.mark.parametrize("precision", [bk.FP32C, bk.FP64])
def test_cv_matches_golden(ctx, name, precision):
    g = load_golden(name)
    kind, dim, h, refs, w = cv_inputs(name)
    wn = w / w.sum()
    ctx.upload(bk.REFERENCE, refs, mass=wn, weight=wn)
    desc = bk.kernel_desc(kind, dim, h)
    lik = ctx.likelihood_cv(desc, precision)
    lsq = ctx.lsq_conv_cv(desc, precision)
    rel = 1e-10 if precision == bk.FP64 else 1e-6
    assert lik == pytest.approx(float(g["likelihood"]), rel=rel)
    assert lsq == pytest.approx(float(g["lsq"]), rel=rel)


def test_cv_adaptive_and_isolated_points(ctx, oracle):
    """LOO after adaptation, and Epanechnikov with an isolated point: its
    leave-one-out density is exactly 0 and the likelihood is -inf, as the
    reference's log(0) gives."""
    rng = W.SplitMix64(77)
    refs = W.f32(rng.normal(4000).reshape(2000, 2) * 0.5)
    w = rng.uniform(2000, 0.5, 1.5)
    wn = w / w.sum()
    ctx.upload(bk.REFERENCE, refs, mass=wn, weight=wn)
    d = bk.kernel_desc(W.GAUSS_PROD2D, 2, (0.1, 0.12))
    abw, mass, _, _ = ctx.adapt_density(d, 0.5, bk.FP64)
    lik = ctx.likelihood_cv(d, bk.FP64)
    want = oracle.likelihood_cv(W.GAUSS_PROD2D, 2, (0.1, 0.12), refs, wn, mass, abw=abw)
    assert lik == pytest.approx(want, rel=1e-10)
    lik32 = ctx.likelihood_cv(d, bk.FP32C)
    assert lik32 == pytest.approx(want, rel=1e-6)
    refs2 = np.vstack([refs, [[50.0, 50.0]]])
    w2 = np.append(wn, 1e-3)
    w2 /= w2.sum()
    ctx.upload(bk.REFERENCE, refs2, mass=w2, weight=w2)
    de = bk.kernel_desc(W.EPAN_PROD2D, 2, (0.3, 0.3))
    assert ctx.likelihood_cv(de, bk.FP32C) == -np.inf
    assert ctx.likelihood_cv(de, bk.FP64) == -np.inf


def test_lsq_requires_a_convolution_kernel(ctx):
    ctx.upload(bk.REFERENCE, np.zeros((4, 2)), mass=np.full(4, 0.25))
    with pytest.raises(bk.BBKDEError):
        ctx.lsq_conv_cv(bk.kernel_desc(W.GAUSS, 2, (0.3,)))   # no 2-D iso conv kernel


@pytest.mark.parametrize("name", sorted(NUMINT_CASES))
def test_lsq_numint_matches_golden(ctx, name):
    """bbkde_lsq_numint_cv against the reference's lsq_numint_cross_validate.
    Tolerance: 2e-6 relative -- FP32-compensated sums (1e-7 per density value,
    culled grid bound 1e-7) in both terms of sq - 2 llo, whose magnitudes are
    close to |cv| here."""
    g = load_golden(name)
    kind, h, alpha, grid, refs, w = numint_inputs(name)
    wn = w / w.sum()
    ctx.upload(bk.REFERENCE, refs, mass=wn, weight=wn)
    desc = bk.kernel_desc(kind, 2, h)
    if alpha >= 0:
        ctx.adapt_density(desc, alpha, bk.FP32C, outputs=False)
    sx, sy, x0, x1, y0, y1 = grid
    got = ctx.lsq_numint_cv(desc, (sx, sy, x0, x1, y0, y1))
    assert got == pytest.approx(float(g["cv"]), rel=2e-6)
    with pytest.raises(bk.BBKDEError):
        ctx.lsq_numint_cv(desc, (sx, sy, x0, x1, y0, y1), precision=bk.FP64)
