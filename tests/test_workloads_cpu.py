"""The seeded generators are deterministic and float32-representable."""
from __future__ import annotations

import numpy as np

from bbrcit_kde_b200 import workloads as W


def test_splitmix_known_values():
    # splitmix64 with state seed + i*golden: first outputs for seed 0.
    r = W.SplitMix64(0)
    v = r.next_u64(3)
    assert [int(x) for x in v] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_open_interval_and_normals():
    r = W.SplitMix64(5)
    u = r.uniform(100000)
    assert u.min() > 0 and u.max() < 1
    z = W.SplitMix64(6).normal(200000)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01


def test_config1_shapes_and_grid():
    wl = W.config1()
    assert wl.refs.shape == (10000, 2) and wl.queries.shape == (10000, 2)
    # generate_2dgrid: x inner, start + i*delta, end excluded
    assert wl.queries[0, 0] == np.float32(-3.0) and wl.queries[1, 0] == np.float32(-3 + 0.06)
    assert wl.queries[100, 1] == np.float32(-3 + 0.06)
    assert wl.queries.max() < 3.0


def test_float32_representable_and_deterministic():
    a = W.config2(n=5000, m=100)
    b = W.config2(n=5000, m=100)
    np.testing.assert_array_equal(a.refs, b.refs)
    np.testing.assert_array_equal(a.refs, a.refs.astype(np.float32).astype(np.float64))
    assert a.weights.min() >= 0.5 and a.weights.max() <= 1.5
    c4 = W.config4(n=4096, m=4096)
    np.testing.assert_array_equal(c4.queries, c4.queries.astype(np.float32).astype(np.float64))
    assert c4.queries.min() >= -6 and c4.queries.max() <= 6


def test_config3_sizes_log_uniform():
    sets = W.config3_datasets(sizes=[100] * 16)
    assert len(sets) == 16 and all(s.shape == (100, 2) for s in sets)
    h = W.config3_bandwidths()
    assert len(h) == 64 and h[0] == 0.01 and abs(h[-1] - 1.0) < 1e-15
