"""Test infrastructure: ctypes bindings for the two CPU checkers.

* ``Oracle``    -- oracle/_build/libkde_oracle.so, the FP64 C restatement.
* ``Reference`` -- oracle/_ref/libkde_ref.so, the reference's own header-only
                   C++ compiled from its sources (see oracle/Makefile).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module. The product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libkde_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libkde_ref.so")

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _c(a, dtype=np.float64):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype)


def build(force: bool = False) -> None:
    """Compile the oracle (and, when the reference headers exist, the harness)."""
    if force or not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", HERE, "all"])


def nthreads_default() -> int:
    return max(1, os.cpu_count() or 1)


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build()
        lib = C.CDLL(path)
        lib.kde_oracle_normalization.restype = C.c_double
        lib.kde_oracle_normalization.argtypes = [C.c_int, C.c_int, _dp]
        lib.kde_oracle_direct.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp, _dp,
                                          C.c_int64, _dp, C.c_int, C.c_int, _dp, C.c_int]
        lib.kde_oracle_self.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp, _dp,
                                        C.c_int, C.c_int, _dp, C.c_int]
        lib.kde_oracle_init_attributes.argtypes = [C.c_int, C.c_int64, _dp, _dp, _dp, _dp]
        lib.kde_oracle_adapt.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp,
                                         C.c_double, _dp, _dp, _dp, _dp, C.c_int]
        lib.kde_oracle_likelihood_cv.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp,
                                                 _dp, _dp, C.c_int, _dp, C.c_int]
        lib.kde_oracle_lsq_conv_cv.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_int64,
                                               _dp, _dp, _dp, _dp, C.c_int, C.c_int, _dp,
                                               C.c_int]
        lib.kde_oracle_lsq_numint_cv.argtypes = [C.c_int, _dp, C.c_int64, _dp, _dp, _dp, _dp,
                                                 C.c_double, C.c_double, C.c_int, C.c_double,
                                                 C.c_double, C.c_int, C.c_int, _dp, C.c_int]
        self.lib = lib

    @staticmethod
    def _h(h):
        h = list(h) + [h[0]] * (2 - len(h))
        return np.asarray(h[:2], dtype=np.float64)

    def normalization(self, kind, dim, h) -> float:
        hh = self._h(h)
        return self.lib.kde_oracle_normalization(kind, dim, _p(hh))

    def direct(self, kind, dim, h, refs, mass, queries, abw=None, normalized=True,
               quirk=True, nthreads=None):
        refs, mass, queries, abw = _c(refs), _c(mass), _c(queries), _c(abw)
        m = queries.shape[0]
        out = np.empty(m)
        hh = self._h(h)
        rc = self.lib.kde_oracle_direct(kind, dim, _p(hh), refs.shape[0], _p(refs), _p(mass),
                                        _p(abw), m, _p(queries), int(normalized), int(quirk),
                                        _p(out), nthreads or nthreads_default())
        assert rc == 0, rc
        return out

    def self_eval(self, kind, dim, h, refs, mass, abw=None, exclude_self=False, quirk=True,
                  nthreads=None):
        refs, mass, abw = _c(refs), _c(mass), _c(abw)
        out = np.empty(refs.shape[0])
        hh = self._h(h)
        rc = self.lib.kde_oracle_self(kind, dim, _p(hh), refs.shape[0], _p(refs), _p(mass),
                                      _p(abw), int(exclude_self), int(quirk), _p(out),
                                      nthreads or nthreads_default())
        assert rc == 0, rc
        return out

    def init_attributes(self, dim, w, abw=None):
        w, abw = _c(w), _c(abw)
        wn = np.empty_like(w)
        mass = np.empty_like(w)
        self.lib.kde_oracle_init_attributes(dim, w.shape[0], _p(w), _p(abw), _p(wn), _p(mass))
        return wn, mass

    def adapt(self, kind, dim, h, refs, w_norm, alpha, nthreads=None):
        refs, w_norm = _c(refs), _c(w_norm)
        n = refs.shape[0]
        pilot, abw, mass, g = np.empty(n), np.empty(n), np.empty(n), np.zeros(1)
        hh = self._h(h)
        rc = self.lib.kde_oracle_adapt(kind, dim, _p(hh), n, _p(refs), _p(w_norm), alpha,
                                       _p(pilot), _p(abw), _p(mass), _p(g),
                                       nthreads or nthreads_default())
        if rc == 2:
            raise ValueError("adapt_density: alpha must be between [0, 1].")
        assert rc == 0, rc
        return pilot, abw, mass, float(g[0])

    def likelihood_cv(self, kind, dim, h, refs, w, mass, abw=None, loo_mode=1, nthreads=None):
        refs, w, mass, abw = _c(refs), _c(w), _c(mass), _c(abw)
        cv = np.zeros(1)
        hh = self._h(h)
        rc = self.lib.kde_oracle_likelihood_cv(kind, dim, _p(hh), refs.shape[0], _p(refs),
                                               _p(w), _p(mass), _p(abw), loo_mode, _p(cv),
                                               nthreads or nthreads_default())
        assert rc == 0, rc
        return float(cv[0])

    def lsq_conv_cv(self, kind, conv_kind, dim, h, refs, w, mass, abw=None, loo_mode=1,
                    quirk=True, nthreads=None):
        refs, w, mass, abw = _c(refs), _c(w), _c(mass), _c(abw)
        cv = np.zeros(1)
        hh = self._h(h)
        rc = self.lib.kde_oracle_lsq_conv_cv(kind, conv_kind, dim, _p(hh), refs.shape[0],
                                             _p(refs), _p(w), _p(mass), _p(abw), loo_mode,
                                             int(quirk), _p(cv), nthreads or nthreads_default())
        assert rc == 0, rc
        return float(cv[0])


    def lsq_numint_cv(self, kind, h, refs, w, mass, grid, abw=None, loo_mode=1, nthreads=None):
        """grid = (steps_x, steps_y, x0, x1, y0, y1)."""
        refs, w, mass, abw = _c(refs), _c(w), _c(mass), _c(abw)
        sx, sy, x0, x1, y0, y1 = grid
        cv = np.zeros(1)
        hh = self._h(h)
        rc = self.lib.kde_oracle_lsq_numint_cv(kind, _p(hh), refs.shape[0], _p(refs), _p(w),
                                               _p(mass), _p(abw), x0, x1, sx, y0, y1, sy,
                                               loo_mode, _p(cv), nthreads or nthreads_default())
        assert rc == 0, rc
        return float(cv[0])


class Reference:
    """The reference's own KernelDensity<> (FP64 CPU), compiled from its headers."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        lib.ref_kde_eval.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp, C.c_double,
                                     C.c_double, C.c_double, C.c_int64, _dp, _dp, _dp, _dp,
                                     _dp, _dp, _i64p, C.c_int]
        lib.ref_kde_likelihood_cv.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp,
                                              C.c_double, C.c_double, C.c_double, _dp]
        lib.ref_kde_lsq_conv_cv.argtypes = lib.ref_kde_likelihood_cv.argtypes
        lib.ref_kde_lsq_numint_cv.argtypes = [C.c_int, _dp, C.c_int64, _dp, _dp, C.c_double,
                                              C.c_double, C.c_double, C.c_int, C.c_double,
                                              C.c_double, C.c_int, C.c_double, C.c_double, _dp]
        lib.ref_kde_normalization.restype = C.c_double
        lib.ref_kde_normalization.argtypes = [C.c_int, C.c_int, _dp]
        lib.ref_kde_create.restype = C.c_void_p
        lib.ref_kde_create.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp]
        lib.ref_kde_direct.argtypes = [C.c_void_p, C.c_int64, _dp, _dp, C.c_int]
        lib.ref_kde_destroy.argtypes = [C.c_void_p]
        lib.ref_kde_tree_eval.argtypes = [C.c_int, C.c_int, _dp, C.c_int64, _dp, _dp,
                                          C.c_double, C.c_double, C.c_double, C.c_int64, _dp,
                                          _dp, _dp, _i64p, _dp, _dp, _dp, _dp, _i64p]
        lib.ref_kde_marginal_direct.argtypes = [C.c_int, _dp, C.c_int64, _dp, _dp, C.c_double,
                                                C.c_double, C.c_double, C.c_int, C.c_int64,
                                                _dp, _dp, _dp, _dp, _dp, _dp, _i64p, C.c_int]
        self.lib = lib

    def create(self, kind, dim, h, refs, w):
        """A persistent KernelDensity<> (Kd-tree built once) for repeated direct_eval."""
        refs, w = _c(refs), _c(w)
        hh = Oracle._h(h)
        handle = self.lib.ref_kde_create(kind, dim, _p(hh), refs.shape[0], _p(refs), _p(w))
        if not handle:
            raise ValueError("unsupported kernel for a persistent handle")
        return handle

    def direct(self, handle, queries, nthreads=None):
        queries = _c(queries)
        out = np.empty(queries.shape[0])
        rc = self.lib.ref_kde_direct(handle, queries.shape[0], _p(queries), _p(out),
                                     nthreads or nthreads_default())
        assert rc == 0, rc
        return out

    def destroy(self, handle):
        self.lib.ref_kde_destroy(handle)

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def normalization(self, kind, dim, h) -> float:
        hh = Oracle._h(h)
        return self.lib.ref_kde_normalization(kind, dim, _p(hh))

    def eval(self, kind, dim, h, refs, w, queries=None, alpha=-1.0, rel=0.0, abs_=0.0,
             nthreads=None):
        """Returns (values at queries, tree-ordered (xy, w, mass, abw))."""
        refs, w = _c(refs), _c(w)
        n = refs.shape[0]
        hh = Oracle._h(h)
        if queries is not None:
            queries = _c(queries)
            m = queries.shape[0]
            out = np.empty(m)
        else:
            m, out = 0, None
        txy, tw, tm, ta = np.empty(n * dim), np.empty(n), np.empty(n), np.empty(n)
        nt = np.zeros(1, dtype=np.int64)
        rc = self.lib.ref_kde_eval(kind, dim, _p(hh), n, _p(refs), _p(w), alpha, rel, abs_,
                                   m, _p(queries), _p(out), _p(txy), _p(tw), _p(tm), _p(ta),
                                   nt.ctypes.data_as(_i64p), nthreads or nthreads_default())
        if rc == 2:
            raise ValueError("invalid argument")
        assert rc == 0, rc
        k = int(nt[0])
        return out, (txy[: k * dim].reshape(k, dim), tw[:k], tm[:k], ta[:k])

    def likelihood_cv(self, kind, dim, h, refs, w, alpha=-1.0, rel=0.0, abs_=0.0):
        refs, w = _c(refs), _c(w)
        cv = np.zeros(1)
        hh = Oracle._h(h)
        rc = self.lib.ref_kde_likelihood_cv(kind, dim, _p(hh), refs.shape[0], _p(refs), _p(w),
                                            alpha, rel, abs_, _p(cv))
        assert rc == 0, rc
        return float(cv[0])

    def lsq_conv_cv(self, kind, dim, h, refs, w, alpha=-1.0, rel=0.0, abs_=0.0):
        refs, w = _c(refs), _c(w)
        cv = np.zeros(1)
        hh = Oracle._h(h)
        rc = self.lib.ref_kde_lsq_conv_cv(kind, dim, _p(hh), refs.shape[0], _p(refs), _p(w),
                                          alpha, rel, abs_, _p(cv))
        assert rc == 0, rc
        return float(cv[0])

    def lsq_numint_cv(self, kind, h, refs, w, grid, alpha=-1.0, rel=0.0, abs_=0.0):
        """The reference's lsq_numint_cross_validate; grid = (steps_x, steps_y, x0, x1,
        y0, y1)."""
        refs, w = _c(refs), _c(w)
        sx, sy, x0, x1, y0, y1 = grid
        cv = np.zeros(1)
        hh = Oracle._h(h)
        rc = self.lib.ref_kde_lsq_numint_cv(kind, _p(hh), refs.shape[0], _p(refs), _p(w),
                                            alpha, x0, x1, sx, y0, y1, sy, rel, abs_, _p(cv))
        assert rc == 0, rc
        return float(cv[0])

    def tree_eval(self, kind, dim, h, refs, w, queries, rel, abs_, alpha=-1.0):
        """The reference's dual-tree eval(queries, rel, abs) after an exact
        adapt_density(alpha) when alpha >= 0. Returns (query coordinates as the
        tree returns them, their values, tree-ordered (xy, w, mass, abw))."""
        refs, w, queries = _c(refs), _c(w), _c(queries)
        n, m = refs.shape[0], queries.shape[0]
        hh = Oracle._h(h)
        oq, out = np.empty(m * dim), np.empty(m)
        mo = np.zeros(1, dtype=np.int64)
        txy, tw, tm, ta = np.empty(n * dim), np.empty(n), np.empty(n), np.empty(n)
        nt = np.zeros(1, dtype=np.int64)
        rc = self.lib.ref_kde_tree_eval(kind, dim, _p(hh), n, _p(refs), _p(w), alpha, rel, abs_,
                                        m, _p(queries), _p(oq), _p(out),
                                        mo.ctypes.data_as(_i64p), _p(txy), _p(tw), _p(tm),
                                        _p(ta), nt.ctypes.data_as(_i64p))
        assert rc == 0, rc
        k, t = int(mo[0]), int(nt[0])
        return (oq[: k * dim].reshape(k, dim), out[:k],
                (txy[: t * dim].reshape(t, dim), tw[:t], tm[:t], ta[:t]))

    def marginal_direct(self, kind, h, refs, w, dim_idx, queries, alpha=-1.0, rel=0.0,
                        abs_=0.0, nthreads=None):
        """The reference's MarginalDensityAssociator marginal of a 2-D product-kernel
        density (after adapt_density(alpha, rel, abs) when alpha >= 0), evaluated by
        direct_eval at 1-D queries. Returns (values, marginal points (x, w, mass,
        abw) in its tree order)."""
        refs, w, queries = _c(refs), _c(w), _c(queries).reshape(-1)
        n, m = refs.shape[0], queries.shape[0]
        hh = Oracle._h(h)
        out = np.empty(m)
        tx, tw, tm, ta = np.empty(n), np.empty(n), np.empty(n), np.empty(n)
        nt = np.zeros(1, dtype=np.int64)
        rc = self.lib.ref_kde_marginal_direct(kind, _p(hh), n, _p(refs), _p(w), alpha, rel,
                                              abs_, dim_idx, m, _p(queries), _p(out), _p(tx),
                                              _p(tw), _p(tm), _p(ta), nt.ctypes.data_as(_i64p),
                                              nthreads or nthreads_default())
        assert rc == 0, rc
        t = int(nt[0])
        return out, (tx[:t], tw[:t], tm[:t], ta[:t])
