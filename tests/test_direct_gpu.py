"""Parity of the CUDA pair sum (through the C ABI) with the reference.

Tolerances:
  FP64  -- rtol 1e-11 against the FP64 oracle / golden vectors (summation order only).
  FP32C -- every entry passes the reference's own CPU-vs-GPU criterion
           approximately_equal(rel 1e-6, abs 1e-8) (FloatUtils.h:49-61,
           test/test_cukde2.cc), with abs scaled by the density's magnitude for
           unnormalised sums.
"""
from __future__ import annotations

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from bbrcit_kde_b200.parity import error_stats
from tests.helpers import PLAIN_CASES, assert_parity, load_golden, plain_inputs

pytestmark = pytest.mark.gpu

REL32, ABS32 = 1e-6, 1e-8


def upload_kde(ctx, refs, w, queries):
    """As KernelDensity does: weights normalised to sum 1, mass = weight, abw = 1."""
    wn = w / w.sum()
    ctx.upload(bk.REFERENCE, refs, mass=wn, abw=None, weight=wn)
    ctx.upload(bk.QUERY, queries)
    return wn


@pytest.mark.parametrize("name", sorted(PLAIN_CASES))
@pytest.mark.parametrize("precision", [bk.FP32C, bk.FP64])
def test_direct_eval_matches_golden(ctx, name, precision):
    g = load_golden(name)
    kind, dim, h, refs, w, q = plain_inputs(name)
    upload_kde(ctx, refs, w, q)
    desc = bk.kernel_desc(kind, dim, h)
    got = ctx.eval_all(desc, normalized=True, precision=precision)
    if precision == bk.FP64:
        np.testing.assert_allclose(got, g["values"], rtol=1e-11, atol=1e-300)
    else:
        assert_parity(got, g["values"], REL32, ABS32, what=name)


KINDS = [(W.GAUSS, 2, (0.2, 0.2)), (W.EPAN, 2, (0.5, 0.5)),
         (W.GAUSS_PROD2D, 2, (0.1, 0.3)), (W.EPAN_PROD2D, 2, (0.4, 0.2)),
         (W.GAUSS_PROD_CONV2D, 2, (0.1, 0.3)), (W.EPAN_PROD_CONV2D, 2, (0.4, 0.2)),
         (W.GAUSS, 1, (0.05, 0.05)), (W.EPAN, 1, (0.2, 0.2)),
         (W.GAUSS_CONV1D, 1, (0.05, 0.05)), (W.EPAN_CONV1D, 1, (0.2, 0.2))]


def _rand_problem(seed, n, m, dim, adaptive=False):
    rng = W.SplitMix64(seed)
    refs = W.f32(rng.normal(n * dim).reshape(n, dim))
    q = W.f32(rng.uniform(m * dim, -3, 3).reshape(m, dim))
    mass = rng.uniform(n, 0.5, 2.0) / n
    abw = rng.uniform(n, 0.5, 2.0) if adaptive else None
    return refs, q, mass, abw


@pytest.mark.parametrize("kind,dim,h", KINDS)
@pytest.mark.parametrize("adaptive", [False, True])
def test_all_kernels_vs_oracle(ctx, oracle, kind, dim, h, adaptive):
    refs, q, mass, abw = _rand_problem(100 + kind * 3 + dim, 3001, 1777, dim, adaptive)
    ctx.upload(bk.REFERENCE, refs, mass=mass, abw=abw)
    ctx.upload(bk.QUERY, q)
    desc = bk.kernel_desc(kind, dim, h)
    want = oracle.direct(kind, dim, h, refs, mass, q, abw=abw)
    got64 = ctx.eval_all(desc, precision=bk.FP64)
    np.testing.assert_allclose(got64, want, rtol=1e-11, atol=1e-300)
    got32 = ctx.eval_all(desc, precision=bk.FP32C)
    assert_parity(got32, want, REL32, ABS32, what=f"kind {kind} dim {dim}")


def test_exact_gauss_conv_flag(ctx, oracle):
    refs, q, mass, _ = _rand_problem(7, 500, 300, 2)
    ctx.upload(bk.REFERENCE, refs, mass=mass)
    ctx.upload(bk.QUERY, q)
    h = (0.2, 0.3)
    for flags, quirk in ((0, True), (bk.FLAG_EXACT_GAUSS_CONV, False)):
        desc = bk.kernel_desc(W.GAUSS_PROD_CONV2D, 2, h, flags)
        want = oracle.direct(W.GAUSS_PROD_CONV2D, 2, h, refs, mass, q, quirk=quirk)
        np.testing.assert_allclose(ctx.eval_all(desc, precision=bk.FP64), want, rtol=1e-11)


@pytest.mark.parametrize("precision", [bk.FP32C, bk.FP64])
def test_closed_subranges_and_unnormalized(ctx, oracle, precision):
    """CudaDirectKde::unnormalized_eval over [r_i, r_j] x [q_i, q_j];
    result[k - q_i] for query k (CudaDirectKde.h:75-88)."""
    refs, q, mass, abw = _rand_problem(11, 5000, 3000, 2, adaptive=True)
    ctx.upload(bk.REFERENCE, refs, mass=mass, abw=abw)
    ctx.upload(bk.QUERY, q)
    h = (0.15, 0.15)
    desc = bk.kernel_desc(W.GAUSS, 2, h)
    for (ri, rj, qi, qj) in [(0, 4999, 0, 2999), (17, 4000, 5, 5), (1234, 1234, 100, 2900),
                             (0, 0, 0, 0), (4999, 4999, 2999, 2999), (300, 2347, 1001, 1500)]:
        got = ctx.eval_range(desc, ri, rj, qi, qj, normalized=False, precision=precision)
        assert got.shape == (qj - qi + 1,)
        want = oracle.direct(W.GAUSS, 2, h, refs[ri:rj + 1], mass[ri:rj + 1], q[qi:qj + 1],
                             abw=abw[ri:rj + 1], normalized=False)
        if precision == bk.FP64:
            np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-300)
        else:
            assert_parity(got, want, REL32, ABS32 * 1e-3, what=str((ri, rj, qi, qj)))


def test_range_errors_match_reference(ctx):
    """CudaDirectKde.h:181-190: j >= size -> out_of_range; i > j -> invalid_argument."""
    refs, q, mass, _ = _rand_problem(3, 100, 50, 2)
    ctx.upload(bk.REFERENCE, refs, mass=mass)
    ctx.upload(bk.QUERY, q)
    d = bk.kernel_desc(W.GAUSS, 2, (0.1,))
    with pytest.raises(bk.OutOfRange):
        ctx.eval_range(d, 0, 100, 0, 49)
    with pytest.raises(bk.OutOfRange):
        ctx.eval_range(d, 0, 99, 0, 50)
    with pytest.raises(bk.InvalidArgument):
        ctx.eval_range(d, 5, 4, 0, 49)
    with pytest.raises(bk.InvalidArgument):
        ctx.eval_range(d, 0, 99, 10, 9)
    with pytest.raises(bk.InvalidArgument):   # kernel dim vs point dim
        ctx.eval_range(bk.kernel_desc(W.GAUSS, 1, (0.1,)), 0, 99, 0, 49)
    with pytest.raises(bk.InvalidArgument):   # product kernels are 2-D only
        ctx.eval_range(bk.kernel_desc(W.GAUSS_PROD2D, 1, (0.1, 0.2)), 0, 99, 0, 49)
    with pytest.raises(bk.InvalidArgument):
        ctx.eval_range(bk.kernel_desc(W.GAUSS, 2, (0.0,)), 0, 99, 0, 49)
    with pytest.raises(bk.InvalidArgument):
        ctx.eval_range(bk.kernel_desc(W.GAUSS, 2, (float("nan"),)), 0, 99, 0, 49)
    with pytest.raises(bk.InvalidArgument):
        ctx.eval_range(bk.kernel_desc(42, 2, (0.1,)), 0, 99, 0, 49)
    with pytest.raises(bk.InvalidArgument):
        ctx.eval_range(d, 0, 99, 0, 49, precision=7)
    # The context stays usable after errors.
    assert ctx.eval_range(d, 0, 99, 0, 49).shape == (50,)


def test_edge_cases(ctx, oracle):
    h = (0.3, 0.3)
    d = bk.kernel_desc(W.GAUSS, 2, h)
    # one reference, one query, query on top of the reference: U(0) = 1 exactly
    ctx.upload(bk.REFERENCE, np.array([[0.25, -0.5]]), mass=np.array([2.0]))
    ctx.upload(bk.QUERY, np.array([[0.25, -0.5]]))
    for p in (bk.FP32C, bk.FP64):
        assert ctx.eval_range(d, 0, 0, 0, 0, normalized=False, precision=p)[0] == 2.0
    # zero masses contribute nothing; far queries underflow to exactly 0
    ctx.upload(bk.REFERENCE, np.array([[0.0, 0.0], [1.0, 1.0]]), mass=np.array([0.0, 1.0]))
    ctx.upload(bk.QUERY, np.array([[1.0, 1.0], [1e4, 1e4]]))
    out = ctx.eval_range(d, 0, 1, 0, 1, normalized=False, precision=bk.FP32C)
    assert out[0] == 1.0 and out[1] == 0.0
    # Epanechnikov: compact support; a point outside every kernel gets exactly 0
    de = bk.kernel_desc(W.EPAN, 2, (0.5,))
    ctx.upload(bk.REFERENCE, np.array([[0.0, 0.0]]), mass=np.array([1.0]))
    ctx.upload(bk.QUERY, np.array([[0.5, 0.0], [0.0, 0.25], [3.0, 3.0]]))
    for p in (bk.FP32C, bk.FP64):
        out = ctx.eval_range(de, 0, 0, 0, 2, normalized=False, precision=p)
        assert out[0] == 0.0 and out[2] == 0.0 and abs(out[1] - 0.75) < 1e-7
    # duplicated references add up like the reference's merged points
    refs = np.array([[0.0, 0.0], [0.0, 0.0], [0.5, 0.5]])
    mass = np.array([0.25, 0.25, 0.5])
    q = np.array([[0.1, 0.1], [0.4, 0.6]])
    ctx.upload(bk.REFERENCE, refs, mass=mass)
    ctx.upload(bk.QUERY, q)
    want = oracle.direct(W.GAUSS, 2, h, refs, mass, q)
    assert_parity(ctx.eval_all(d, precision=bk.FP32C), want, REL32, ABS32)


def test_ragged_sizes(ctx, oracle):
    """Sizes around the tile / block / segment boundaries."""
    h = (0.3,)
    d = bk.kernel_desc(W.GAUSS, 1, h)
    for n, m in [(1, 1), (31, 33), (255, 257), (256, 1024), (513, 1025), (4097, 1),
                 (1, 4097), (70001, 3)]:
        refs, q, mass, _ = _rand_problem(n * 7 + m, n, m, 1)
        ctx.upload(bk.REFERENCE, refs, mass=mass)
        ctx.upload(bk.QUERY, q)
        want = oracle.direct(W.GAUSS, 1, h, refs, mass, q)
        np.testing.assert_allclose(ctx.eval_all(d, precision=bk.FP64), want, rtol=1e-11,
                                   atol=1e-300)
        assert_parity(ctx.eval_all(d, precision=bk.FP32C), want, REL32, ABS32,
                      what=f"n={n} m={m}")


def test_deterministic_bitwise(ctx):
    refs, q, mass, abw = _rand_problem(5, 20000, 7000, 2, adaptive=True)
    ctx.upload(bk.REFERENCE, refs, mass=mass, abw=abw)
    ctx.upload(bk.QUERY, q)
    d = bk.kernel_desc(W.GAUSS_PROD2D, 2, (0.05, 0.08))
    a = ctx.eval_all(d, precision=bk.FP32C)
    b = ctx.eval_all(d, precision=bk.FP32C)
    np.testing.assert_array_equal(a, b)


def test_launch_stats(ctx):
    refs, q, mass, _ = _rand_problem(9, 4096, 8192, 2)
    ctx.upload(bk.REFERENCE, refs, mass=mass)
    ctx.upload(bk.QUERY, q)
    ctx.eval_all(bk.kernel_desc(W.GAUSS, 2, (0.1,)))
    ms, pairs, launches = ctx.last_launch_stats()
    assert pairs == 4096 * 8192 and ms > 0 and launches >= 1


def test_config2_full_size_properties(ctx, oracle):
    """1M x 1M refs/queries of the adaptive-product-Gaussian workload: FP32C vs
    the FP64 device path on a 4096-query slice, the CPU oracle on 256 queries,
    and linearity over a split of the reference range."""
    wl = W.config2()
    wn = wl.weights / wl.weights.sum()
    n = len(wl.refs)
    rng = W.SplitMix64(99)
    abw = rng.uniform(n, 0.5, 3.0)
    mass = wn * abw ** -2
    ctx.upload(bk.REFERENCE, wl.refs, mass=mass, abw=abw, weight=wn)
    ctx.upload(bk.QUERY, wl.queries)
    d = bk.kernel_desc(W.GAUSS_PROD2D, 2, wl.h)
    qi, qj = 500_000, 500_000 + 4095
    f32 = ctx.eval_range(d, 0, n - 1, qi, qj, precision=bk.FP32C)
    f64 = ctx.eval_range(d, 0, n - 1, qi, qj, precision=bk.FP64)
    assert_parity(f32, f64, REL32, ABS32, what="fp32c vs fp64 device")
    want = oracle.direct(W.GAUSS_PROD2D, 2, wl.h, wl.refs, mass, wl.queries[qi:qi + 256],
                         abw=abw)
    np.testing.assert_allclose(f64[:256], want, rtol=1e-10)
    half = n // 2
    lo = ctx.eval_range(d, 0, half - 1, qi, qj, precision=bk.FP64)
    hi = ctx.eval_range(d, half, n - 1, qi, qj, precision=bk.FP64)
    np.testing.assert_allclose(lo + hi, f64, rtol=1e-12)


@pytest.mark.parametrize("kind,dim,h", [(W.GAUSS, 2, (0.2, 0.2)), (W.GAUSS_PROD2D, 2, (0.1, 0.3)),
                                        (W.EPAN_PROD2D, 2, (0.4, 0.2)), (W.GAUSS, 1, (0.05,)),
                                        (W.EPAN_PROD_CONV2D, 2, (0.4, 0.2))])
def test_every_launch_variant(ctx, oracle, kind, dim, h):
    """Each FP32 launch shape the autotuner may pick (including those that put every
    4th, 8th, 16th or 32nd reference's exponentials on the FP32 pipe) gives the same parity,
    including the self-evaluation diagonal exclusion."""
    refs, q, mass, abw = _rand_problem(31 + kind, 5003, 4099, dim, adaptive=True)
    desc = bk.kernel_desc(kind, dim, h)
    want = oracle.direct(kind, dim, h, refs, mass, q, abw=abw)
    want_self = oracle.self_eval(kind, dim, h, refs, mass, abw=abw, exclude_self=True)
    with np.errstate(divide="ignore"):   # an isolated point: log(0) = -inf on both sides
        want_lik = np.sum(mass * np.log(want_self))
    n, _ = ctx.launch_variants()
    assert n == 11
    try:
        for v in range(n):
            ctx.set_launch_variant(v)
            ctx.upload(bk.REFERENCE, refs, mass=mass, abw=abw, weight=mass)
            ctx.upload(bk.QUERY, q)
            assert_parity(ctx.eval_all(desc), want, REL32, ABS32, what=f"variant {v}")
            assert ctx.launch_variants()[1] == v
            ctx.upload(bk.QUERY, refs)
            lik = ctx.likelihood_cv(desc)
            np.testing.assert_allclose(lik, want_lik, rtol=1e-6)
        with pytest.raises(bk.InvalidArgument):
            ctx.set_launch_variant(n)
    finally:
        ctx.set_launch_variant(-1)
