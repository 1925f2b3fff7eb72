"""Seeded synthetic inputs for the five benchmark workloads.

The reference has no datasets of its own; its demos draw from libstdc++'s
``std::normal_distribution`` (test/kde_test_utils.h:30-77), whose stream is
implementation-specific. These generators use splitmix64 and Box-Muller instead,
so the CUDA library, the FP64 oracle and the reference harness all see the very
same numbers on any machine.

Every coordinate is rounded to the nearest float32 and stored as the float64 of
that float32, so the FP32 device path and the FP64 checkers start from identical
inputs. Grids follow the reference's ``generate_2dgrid`` (test/kde_test_utils.h:
97-123): ``start + i * (end - start) / steps``, end point excluded, y outer.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)

SEED_BASE = 0xB2000000


class SplitMix64:
    """Counter-based splitmix64: draw i returns mix(seed + (i+1) * golden)."""

    def __init__(self, seed: int):
        self.seed = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        self.counter = 0

    def next_u64(self, n: int) -> np.ndarray:
        i = np.arange(self.counter + 1, self.counter + n + 1, dtype=np.uint64)
        self.counter += n
        with np.errstate(over="ignore"):
            z = self.seed + i * _GOLDEN
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))

    def uniform(self, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
        """Doubles in the open interval (lo, hi)."""
        u = ((self.next_u64(n) >> np.uint64(11)).astype(np.float64) + 0.5) * (2.0 ** -53)
        return lo + (hi - lo) * u

    def normal(self, n: int) -> np.ndarray:
        """Box-Muller standard normals (cosine branch of each pair)."""
        u1 = self.uniform(n)
        u2 = self.uniform(n)
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def f32(a) -> np.ndarray:
    """Round to float32 and return the exact float64 of that float32."""
    return np.asarray(a, dtype=np.float64).astype(np.float32).astype(np.float64)


def grid_2d(start_x, end_x, steps_x, start_y, end_y, steps_y) -> np.ndarray:
    """test/kde_test_utils.h:97-123 (y outer, x inner, end point excluded)."""
    dx = (end_x - start_x) / steps_x
    dy = (end_y - start_y) / steps_y
    ys = start_y + np.arange(steps_y) * dy
    xs = start_x + np.arange(steps_x) * dx
    gx, gy = np.meshgrid(xs, ys)
    return f32(np.stack([gx.ravel(), gy.ravel()], axis=1))


def bimodal_2d(rng: SplitMix64, n: int, means=((-1.0, -1.0), (1.0, 1.0)),
               sigma=0.5, p1=0.5) -> np.ndarray:
    comp = rng.uniform(n) < p1
    zx = rng.normal(n)
    zy = rng.normal(n)
    mx = np.where(comp, means[0][0], means[1][0])
    my = np.where(comp, means[0][1], means[1][1])
    return f32(np.stack([mx + sigma * zx, my + sigma * zy], axis=1))


def mixture_2d_iso(rng: SplitMix64, n: int, means: np.ndarray, sigmas: np.ndarray) -> np.ndarray:
    k = len(means)
    comp = np.minimum((rng.uniform(n) * k).astype(np.int64), k - 1)
    zx = rng.normal(n)
    zy = rng.normal(n)
    return f32(np.stack([means[comp, 0] + sigmas[comp] * zx,
                         means[comp, 1] + sigmas[comp] * zy], axis=1))


@dataclass
class Workload:
    name: str
    kind: int                 # bbkde kernel kind
    dim: int
    h: tuple
    refs: np.ndarray          # (n, dim) float64, float32-representable
    weights: np.ndarray       # (n,) raw (unnormalised) weights
    queries: np.ndarray       # (m, dim)
    alpha: float = -1.0       # < 0: not adaptive
    extra: dict = field(default_factory=dict)


# Kernel kinds (include/bbkde.h).
GAUSS, EPAN, GAUSS_PROD2D, EPAN_PROD2D = 0, 1, 2, 3
GAUSS_PROD_CONV2D, EPAN_PROD_CONV2D, GAUSS_CONV1D, EPAN_CONV1D = 4, 5, 6, 7


def config1(n: int = 10_000, steps: int = 100) -> Workload:
    """Plain 2-D Gaussian, h = 0.1, bimodal refs, 100x100 grid over [-3,3)^2."""
    rng = SplitMix64(SEED_BASE + 1)
    refs = bimodal_2d(rng, n)
    q = grid_2d(-3.0, 3.0, steps, -3.0, 3.0, steps)
    return Workload("plain_gauss2d_n10k_grid100", GAUSS, 2, (0.1, 0.1), refs,
                    np.ones(n), q)


def config2(n: int = 1_000_000, m: int = 1_000_000) -> Workload:
    """Adaptive product Gaussian, pilot (0.05, 0.05), alpha 0.5, weights U[0.5,1.5]."""
    rng = SplitMix64(SEED_BASE + 2)
    refs = bimodal_2d(rng, n)
    w = rng.uniform(n, 0.5, 1.5)
    q = f32(rng.uniform(2 * m, -3.0, 3.0).reshape(m, 2))
    return Workload(f"adaptive_gaussprod2d_n{n}_m{m}", GAUSS_PROD2D, 2, (0.05, 0.05),
                    refs, w, q, alpha=0.5)


def config3_datasets(n_sets: int = 16, n_lo: float = 1e4, n_hi: float = 5e5,
                     sizes=None):
    """16 datasets of log-uniform size, 3-component isotropic mixtures."""
    rng = SplitMix64(SEED_BASE + 3)
    out = []
    for d in range(n_sets):
        nd = int(math.floor(math.exp(rng.uniform(1, math.log(n_lo), math.log(n_hi))[0])))
        if sizes is not None:
            nd = int(sizes[d])
        means = rng.uniform(6, -2.0, 2.0).reshape(3, 2)
        sig = rng.uniform(3, 0.2, 0.8)
        out.append(mixture_2d_iso(rng, nd, means, sig))
    return out


def config3_bandwidths(n: int = 64) -> np.ndarray:
    """h_a = 0.01 * 100^(a/(n-1)), a = 0..n-1 (log-spaced over [0.01, 1])."""
    return 0.01 * 100.0 ** (np.arange(n) / (n - 1))


def config4(n: int = 1 << 24, m: int = 1 << 24) -> Workload:
    """1-D Gaussian, h = 0.02, 5-component mixture, queries U[-6, 6]."""
    rng = SplitMix64(SEED_BASE + 4)
    means = rng.uniform(5, -5.0, 5.0)
    sig = rng.uniform(5, 0.1, 1.0)
    comp = np.minimum((rng.uniform(n) * 5).astype(np.int64), 4)
    refs = f32(means[comp] + sig[comp] * rng.normal(n)).reshape(n, 1)
    q = f32(rng.uniform(m, -6.0, 6.0)).reshape(m, 1)
    return Workload(f"gauss1d_n{n}_m{m}", GAUSS, 1, (0.02,), refs, np.ones(n), q)


def config5_refs(n: int = 4_000_000) -> np.ndarray:
    """8-component 2-D mixture with random SPD covariances (eigenvalues U[0.05,0.5])."""
    rng = SplitMix64(SEED_BASE + 5)
    means = rng.uniform(16, -3.0, 3.0).reshape(8, 2)
    lam = rng.uniform(16, 0.05, 0.5).reshape(8, 2)
    th = rng.uniform(8, 0.0, 2.0 * math.pi)
    comp = np.minimum((rng.uniform(n) * 8).astype(np.int64), 7)
    z1 = rng.normal(n) * np.sqrt(lam[comp, 0])
    z2 = rng.normal(n) * np.sqrt(lam[comp, 1])
    c, s = np.cos(th[comp]), np.sin(th[comp])
    return f32(np.stack([means[comp, 0] + c * z1 - s * z2,
                         means[comp, 1] + s * z1 + c * z2], axis=1))
