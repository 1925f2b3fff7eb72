"""The surrogate's BF16 tensor-core kernels against the FP64 restatement
(tests/mlp_ref.py): forward values, gradients, training, checkpoints."""
from __future__ import annotations

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from tests import mlp_ref

pytestmark = pytest.mark.gpu


def _norm_inputs(xy, norm):
    return np.stack([(xy[:, 0] - norm[0]) * norm[2], (xy[:, 1] - norm[1]) * norm[3]], 1)


def _smooth_target(xy):
    """log of a two-component Gaussian mixture: a smooth log-density."""
    d1 = np.exp(-0.5 * ((xy[:, 0] + 1) ** 2 + (xy[:, 1] + 1) ** 2) / 0.25)
    d2 = np.exp(-0.5 * ((xy[:, 0] - 1) ** 2 + (xy[:, 1] - 1.2) ** 2) / 0.4)
    return np.log(0.3 * d1 + 0.7 * d2 + 1e-2)


def test_forward_matches_fp64_with_bf16_rounding():
    s = bk.Surrogate(0, seed=3)
    p, norm = s.params()
    xy = W.SplitMix64(5).uniform(2 * 3001, -4, 4).reshape(-1, 2)
    got = s.predict(xy)
    y, _ = mlp_ref.forward(p.astype(np.float64), _norm_inputs(xy, norm), emulate_bf16=True)
    want = norm[4] + norm[5] * y
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-3 * (np.abs(want).max() + 1))


@pytest.mark.parametrize("split", [False, True])
def test_tcgen05_inference_matches_mma_sync_and_fp64(split):
    """The tcgen05 (TMEM) inference kernel against the mma.sync kernel and the
    FP64 restatement. Tolerances: with BF16 activations a last-bit difference in
    an FP32 accumulator can flip one BF16 rounding (2^-9 relative on one
    activation), so the engines agree to 2e-3 of the output scale as the FP64
    check does; with two-term activations (rounding ~2^-17) to 1e-4."""
    s = bk.Surrogate(0, seed=5)
    s.set_inference(split)
    p, norm = s.params()
    rng = W.SplitMix64(15)
    xy = rng.uniform(2 * 5003, -4, 4).reshape(-1, 2)      # ragged: 39 tiles + 11 points
    s.set_engine(bk.ENGINE_TCGEN05)
    tc = s.predict(xy)
    s.set_engine(bk.ENGINE_MMA_SYNC)
    ms = s.predict(xy)
    scale = np.abs(ms).max() + 1
    tol = 1e-4 if split else 2e-3
    np.testing.assert_allclose(tc, ms, rtol=0, atol=tol * scale)
    y, _ = mlp_ref.forward(p.astype(np.float64), _norm_inputs(xy, norm), emulate_bf16=not split,
                           bf16_weights=True)
    want = norm[4] + norm[5] * y
    np.testing.assert_allclose(tc, want, rtol=0, atol=2e-3 * scale)


@pytest.mark.parametrize("n", [1000, 128, 300])
def test_tcgen05_gradient_matches_fp64_with_its_rounding(n):
    """The tcgen05 training step's gradient (the default engine) against the FP64
    restatement with the same BF16 rounding points (mlp_ref.loss_and_grad_tc):
    what is left is FP32 against FP64 accumulation, the fast SiLU, and the rare
    BF16 rounding that an FP32 last-bit difference moves. Every parameter block
    within 1e-3 of its norm; ragged point counts leave partial 128-point tiles."""
    s = bk.Surrogate(0, seed=11)
    s.set_engine(bk.ENGINE_TCGEN05)
    p, norm = s.params()
    rng = W.SplitMix64(9 + n)
    xy = rng.uniform(2 * n, -3, 3).reshape(-1, 2)
    t = _smooth_target(xy)
    g, loss = s.gradient(xy, t)
    xin = _norm_inputs(xy, norm)
    tn = (t - norm[4]) / norm[5]
    loss64, g64 = mlp_ref.loss_and_grad_tc(p.astype(np.float64), xin, tn)
    assert loss == pytest.approx(loss64, rel=1e-5)
    for name, (o, k) in mlp_ref.OFF.items():
        a, b = g[o:o + k], g64[o:o + k]
        assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b) + 1e-9, \
            (name, np.linalg.norm(a - b) / np.linalg.norm(b))
    # deterministic: the same call gives the same bits
    g2, loss2 = s.gradient(xy, t)
    np.testing.assert_array_equal(g2, g)
    assert loss2 == loss


def test_training_engines_agree():
    """Training on tcgen05 and on mma.sync from the same start reaches the same
    held-out error scale (their rounding points differ, so not the same bits)."""
    rng = W.SplitMix64(31)
    xy = rng.uniform(2 * 100_000, -3, 3).reshape(-1, 2)
    t = _smooth_target(xy)
    test_xy = W.SplitMix64(32).uniform(2 * 10_000, -3, 3).reshape(-1, 2)
    test_t = _smooth_target(test_xy)
    errs = []
    for engine in (bk.ENGINE_TCGEN05, bk.ENGINE_MMA_SYNC):
        s = bk.Surrogate(0, seed=4)
        s.set_engine(engine)
        s.train(xy, t, steps=1500, batch=8192, lr=3e-3, lr_final=1e-5)
        errs.append(float(np.median(np.abs(s.predict(test_xy) - test_t))))
    assert errs[0] < 0.05 and errs[1] < 0.05, errs
    assert 0.5 < errs[0] / errs[1] < 2.0, errs


def test_gradient_matches_fp64_backprop():
    """The legacy mma.sync training engine, which also stores pre-activations and
    gradients in BF16: against the restatement with forward rounding only."""
    s = bk.Surrogate(0, seed=11)
    s.set_engine(bk.ENGINE_MMA_SYNC)
    p, norm = s.params()
    rng = W.SplitMix64(9)
    xy = rng.uniform(2 * 1000, -3, 3).reshape(-1, 2)
    t = _smooth_target(xy)
    g, loss = s.gradient(xy, t)
    _, norm = s.params()                 # unchanged by gradient()
    xin = _norm_inputs(xy, norm)
    tn = (t - norm[4]) / norm[5]
    loss64, g64 = mlp_ref.loss_and_grad(p.astype(np.float64), xin, tn, emulate_bf16=True)
    assert loss == pytest.approx(loss64, rel=1e-2)
    cos = float(g @ g64 / (np.linalg.norm(g) * np.linalg.norm(g64)))
    rel = float(np.linalg.norm(g - g64) / np.linalg.norm(g64))
    assert cos > 0.9995 and rel < 3e-2, (cos, rel)
    # every parameter block individually
    for name, (o, n) in mlp_ref.OFF.items():
        a, b = g[o:o + n], g64[o:o + n]
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-7, name


def test_training_reduces_error_and_checkpoint_roundtrip(tmp_path):
    s = bk.Surrogate(0, seed=1)
    rng = W.SplitMix64(21)
    xy = rng.uniform(2 * 200_000, -3, 3).reshape(-1, 2)
    t = _smooth_target(xy)
    test_xy = W.SplitMix64(22).uniform(2 * 20_000, -3, 3).reshape(-1, 2)
    test_t = _smooth_target(test_xy)
    err0 = np.abs(s.predict(test_xy) - test_t)
    _, loss0 = s.gradient(test_xy, test_t)
    s.train(xy, t, steps=4000, batch=8192, lr=3e-3, lr_final=1e-5)
    # loss of the trained network on held-out points (normalisation fixed by training)
    _, loss1 = s.gradient(test_xy, test_t)
    err = np.abs(s.predict(test_xy) - test_t)
    assert loss1 < 1e-2 * loss0 and np.median(err) < 0.02 and err.max() < 0.1 * err0.max(), \
        (loss0, loss1, err0.max(), err.max(), np.median(err))
    path = tmp_path / "s.bbkde"
    s.save(path)
    s2 = bk.Surrogate(0, seed=99)
    s2.load(path)
    np.testing.assert_array_equal(s2.predict(test_xy), s.predict(test_xy))
    with pytest.raises(bk.InvalidArgument):
        s2.load(tmp_path / "missing.bbkde")
