"""The FP64 oracle (oracle/kde_oracle.c) pinned against the reference.

Two pins: the committed golden vectors (made by the reference's own code, see
tests/golden/make_golden.py), and, where the reference harness is built, a live
comparison with the reference on fresh seeded inputs.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from bbrcit_kde_b200 import workloads as W
from tests.helpers import (ADAPTIVE_CASES, CV_CASES, NUMINT_CASES, PLAIN_CASES, adaptive_inputs,
                           cv_inputs, numint_inputs,
                           digest, load_golden, match_by_coords, plain_inputs)

TOL = 1e-12   # FP64 vs FP64: only summation order differs


@pytest.mark.parametrize("name", sorted(PLAIN_CASES))
def test_oracle_direct_matches_golden(oracle, name):
    g = load_golden(name)
    kind, dim, h, refs, w, q = plain_inputs(name)
    assert digest(refs, w, q) == str(g["input_digest"]), "seeded inputs changed"
    wn, mass = oracle.init_attributes(dim, w)
    got = oracle.direct(kind, dim, h, refs, mass, q)
    np.testing.assert_allclose(got, g["values"], rtol=TOL, atol=1e-300)
    assert oracle.normalization(kind, dim, h) == pytest.approx(float(g["normalization"]),
                                                               rel=1e-15)


@pytest.mark.parametrize("name", sorted(ADAPTIVE_CASES))
def test_oracle_adapt_matches_golden(oracle, name):
    g = load_golden(name)
    kind, dim, h, refs, w, q = adaptive_inputs(name)
    assert digest(refs, w, q) == str(g["input_digest"])
    wn, _ = oracle.init_attributes(dim, w)
    pilot, abw, mass, gm = oracle.adapt(kind, dim, h, refs, wn, 0.5)
    # The reference stores per-point results in Kd-tree order: match by coordinates.
    pa, pb = match_by_coords(refs, g["tree_xy"].reshape(-1, dim))
    np.testing.assert_allclose(abw[pa], g["tree_abw"][pb], rtol=1e-10)
    np.testing.assert_allclose(mass[pa], g["tree_mass"][pb], rtol=1e-10)
    np.testing.assert_allclose(wn[pa], g["tree_w"][pb], rtol=1e-14)
    got = oracle.direct(kind, dim, h, refs, mass, q, abw=abw)
    np.testing.assert_allclose(got, g["values"], rtol=1e-9)


@pytest.mark.parametrize("name", sorted(CV_CASES))
def test_oracle_cv_matches_golden(oracle, name):
    g = load_golden(name)
    kind, dim, h, refs, w = cv_inputs(name)
    assert digest(refs, w) == str(g["input_digest"])
    wn, mass = oracle.init_attributes(dim, w)
    conv = {W.GAUSS: W.GAUSS_CONV1D, W.EPAN: W.EPAN_CONV1D,
            W.GAUSS_PROD2D: W.GAUSS_PROD_CONV2D, W.EPAN_PROD2D: W.EPAN_PROD_CONV2D}[kind]
    for loo_mode in (0, 1):   # subtract the self term (reference) / exclude it
        lik = oracle.likelihood_cv(kind, dim, h, refs, wn, mass, loo_mode=loo_mode)
        lsq = oracle.lsq_conv_cv(kind, conv, dim, h, refs, wn, mass, loo_mode=loo_mode)
        assert lik == pytest.approx(float(g["likelihood"]), rel=1e-11)
        assert lsq == pytest.approx(float(g["lsq"]), rel=1e-11)


def test_normalization_known_answers(oracle):
    """test/test_kernels.cc prints these next to their closed forms ("c.f.")."""
    one = (1.0, 1.0)
    assert oracle.normalization(W.GAUSS, 1, one) == pytest.approx(1 / math.sqrt(2 * math.pi))
    assert oracle.normalization(W.GAUSS, 2, one) == pytest.approx(1 / (2 * math.pi))
    assert oracle.normalization(W.EPAN, 1, one) == pytest.approx(0.75)
    assert oracle.normalization(W.EPAN, 2, one) == pytest.approx(2 / math.pi)
    assert oracle.normalization(W.GAUSS_PROD2D, 2, one) == pytest.approx(1 / (2 * math.pi))
    assert oracle.normalization(W.EPAN_PROD2D, 2, one) == pytest.approx(0.5625)
    assert oracle.normalization(W.GAUSS_PROD_CONV2D, 2, one) == pytest.approx(1 / (4 * math.pi))
    assert oracle.normalization(W.EPAN_PROD_CONV2D, 2, one) == pytest.approx(0.36)
    # GaussianTraits<1,double>::normalization takes a float bandwidth
    # (KernelTraits.h:143): h = 0.02 is rounded to float first.
    c = oracle.normalization(W.GAUSS, 1, (0.02, 0.02))
    assert c == 0.3989422804014326779 / float(np.float32(0.02))
    assert c != 0.3989422804014326779 / 0.02


def test_kernels_integrate_to_one(oracle):
    """Normalised kernels integrate to 1 (midpoint rule), except the reference's
    product Gaussian convolution kernel, whose exp(-0.5 arg) quirk
    (KernelTraits.h:444-446) makes it integrate to 1/2."""
    xs = np.linspace(-6, 6, 1201)[:-1] + 0.005
    one = np.zeros((1, 1))
    for kind, h in [(W.GAUSS, 0.7), (W.EPAN, 0.7), (W.GAUSS_CONV1D, 0.7), (W.EPAN_CONV1D, 0.7)]:
        vals = oracle.direct(kind, 1, (h, h), one, np.ones(1), xs.reshape(-1, 1))
        assert vals.sum() * 0.01 == pytest.approx(1.0, abs=2e-4), kind
    g = np.stack(np.meshgrid(xs[::4], xs[::4]), -1).reshape(-1, 2)
    one2 = np.zeros((1, 2))
    for kind, target in [(W.GAUSS, 1.0), (W.EPAN, 1.0), (W.GAUSS_PROD2D, 1.0),
                         (W.EPAN_PROD2D, 1.0), (W.EPAN_PROD_CONV2D, 1.0),
                         (W.GAUSS_PROD_CONV2D, 0.5)]:
        vals = oracle.direct(kind, 2, (0.7, 0.9), one2, np.ones(1), g)
        assert vals.sum() * 0.04 ** 2 == pytest.approx(target, rel=5e-3), kind
    vals = oracle.direct(W.GAUSS_PROD_CONV2D, 2, (0.7, 0.9), one2, np.ones(1), g, quirk=False)
    assert vals.sum() * 0.04 ** 2 == pytest.approx(1.0, rel=5e-3)


@pytest.mark.parametrize("name", sorted(NUMINT_CASES))
@pytest.mark.parametrize("loo_mode", [0, 1])
def test_oracle_lsq_numint_matches_golden(oracle, name, loo_mode):
    """lsq_numint_cross_validate (KernelDensityImpl.h:14-97) against the value the
    reference's own function produced (tests/golden/make_golden.py)."""
    g = load_golden(name)
    kind, h, alpha, grid, refs, w = numint_inputs(name)
    assert g["input_digest"] == digest(refs, w)
    wn = w / w.sum()
    mass, abw = wn, None
    if alpha >= 0:
        _, abw, mass, _ = oracle.adapt(kind, 2, h, refs, wn, alpha)
    got = oracle.lsq_numint_cv(kind, h, refs, wn, mass, grid, abw=abw, loo_mode=loo_mode)
    assert got == pytest.approx(float(g["cv"]), rel=1e-10)


def test_adapt_rejects_bad_alpha(oracle):
    refs = np.zeros((3, 2))
    w = np.full(3, 1 / 3)
    for alpha in (-0.1, 1.5):
        with pytest.raises(ValueError):
            oracle.adapt(W.GAUSS, 2, (1.0, 1.0), refs, w, alpha)


KINDS_LIVE = [(W.GAUSS, 2, (0.2, 0.2)), (W.EPAN, 2, (0.5, 0.5)),
              (W.GAUSS_PROD2D, 2, (0.1, 0.3)), (W.EPAN_PROD2D, 2, (0.4, 0.2)),
              (W.GAUSS_PROD_CONV2D, 2, (0.1, 0.3)), (W.EPAN_PROD_CONV2D, 2, (0.4, 0.2)),
              (W.GAUSS, 1, (0.05, 0.05)), (W.EPAN, 1, (0.2, 0.2)),
              (W.GAUSS_CONV1D, 1, (0.05, 0.05)), (W.EPAN_CONV1D, 1, (0.2, 0.2))]


@pytest.mark.parametrize("kind,dim,h", KINDS_LIVE)
def test_oracle_vs_reference_live(oracle, reference, kind, dim, h):
    rng = W.SplitMix64(1234 + kind * 7 + dim)
    refs = W.f32(rng.normal(700 * dim).reshape(700, dim))
    q = W.f32(rng.uniform(300 * dim, -3, 3).reshape(300, dim))
    w = rng.uniform(700, 0.5, 2.0)
    want, _ = reference.eval(kind, dim, h, refs, w, q)
    wn, mass = oracle.init_attributes(dim, w)
    got = oracle.direct(kind, dim, h, refs, mass, q)
    np.testing.assert_allclose(got, want, rtol=TOL, atol=1e-300)


def test_oracle_merges_nothing_but_reference_does(oracle, reference):
    """The reference's Kd-tree merges exact duplicates (Kdtree.h:365-390); for a
    direct sum that is invisible, so both agree on duplicated inputs."""
    refs = np.array([[0.0, 0.0], [0.0, 0.0], [1.0, 0.5], [1.0, 0.5], [2.0, 2.0]])
    w = np.array([1.0, 2.0, 1.0, 1.0, 3.0])
    q = np.array([[0.1, 0.2], [1.5, 1.5]])
    want, (txy, tw, tm, ta) = reference.eval(W.GAUSS, 2, (0.5, 0.5), refs, w, q)
    assert len(tw) == 3   # merged
    wn, mass = oracle.init_attributes(2, w)
    got = oracle.direct(W.GAUSS, 2, (0.5, 0.5), refs, mass, q)
    np.testing.assert_allclose(got, want, rtol=1e-14)
