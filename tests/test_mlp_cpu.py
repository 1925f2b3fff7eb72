"""The FP64 restatement of the surrogate network is itself checked by central
finite differences (CPU only)."""
from __future__ import annotations

import numpy as np

from tests import mlp_ref


def test_backprop_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(size=mlp_ref.N_PARAMS) * 0.1
    x = rng.uniform(-1, 1, size=(37, 2))
    t = rng.normal(size=37)
    loss, g = mlp_ref.loss_and_grad(p, x, t)
    idx = np.concatenate([rng.choice(n, 6, replace=False) + o
                          for (o, n) in mlp_ref.OFF.values() if n > 1] + [[mlp_ref.OFF["b4"][0]]])
    eps = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mlp_ref.loss_and_grad(pp, x, t)[0] - mlp_ref.loss_and_grad(pm, x, t)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_helper():
    v = np.array([1.0, 1.0 + 2 ** -9, 1.0 + 2 ** -7, -3.140625, 1e-40])
    r = mlp_ref.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7 and r[3] == -3.140625
