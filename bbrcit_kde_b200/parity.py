"""Error statistics of a device result against an FP64 result.

One definition is used everywhere a result is reported (tests, bench.py):

* ``pass_rate``: fraction of entries that satisfy the reference's own
  CPU-vs-GPU criterion ``approximately_equal(lhs, rhs, rel_err, abs_err)``
  (FloatUtils.h:49-61; test/test_cukde2.cc uses rel 1e-6, abs 1e-8): pass iff
  |a - b| <= abs_err or |a - b| <= rel_err * max(|a|, |b|).
* ``max_rel_sig``: max relative error over entries with |ref| >= 1e-6 max|ref|.
* ``max_rel_1e3``: max relative error over entries with |ref| >= 1e-3 max|ref|.
* ``max_abs_over_max``: max |a - b| / max|ref| over all entries.
"""
from __future__ import annotations

import numpy as np


def approximately_equal(a, b, rel_err=1e-6, abs_err=1e-8):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.abs(a - b)
    both_inf = np.isinf(a) & np.isinf(b) & (np.sign(a) == np.sign(b))
    return both_inf | (d <= abs_err) | (d <= rel_err * np.maximum(np.abs(a), np.abs(b)))


def error_stats(got, ref, rel_err=1e-6, abs_err=1e-8) -> dict:
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if got.size == 0:
        return dict(n=0, pass_rate=1.0, n_fail=0, max_rel_sig=0.0, max_rel_1e3=0.0,
                    max_abs_over_max=0.0, median_rel=0.0, rel_err=rel_err, abs_err=abs_err)
    ok = approximately_equal(got, ref, rel_err, abs_err)
    d = np.abs(got - ref)
    fmax = float(np.max(np.abs(ref))) if np.isfinite(ref).any() else 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        rel = np.where(np.abs(ref) > 0, d / np.abs(ref), np.where(d > 0, np.inf, 0.0))
    sig = np.abs(ref) >= 1e-6 * fmax
    sig3 = np.abs(ref) >= 1e-3 * fmax
    return dict(
        n=int(got.size),
        pass_rate=float(ok.mean()),
        n_fail=int((~ok).sum()),
        max_rel_sig=float(rel[sig].max()) if sig.any() else 0.0,
        max_rel_1e3=float(rel[sig3].max()) if sig3.any() else 0.0,
        max_abs_over_max=float(d.max() / fmax) if fmax > 0 else float(d.max()),
        median_rel=float(np.median(rel[sig])) if sig.any() else 0.0,
        rel_err=rel_err, abs_err=abs_err,
    )
