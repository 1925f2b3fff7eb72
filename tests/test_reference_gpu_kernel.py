"""The reference's own GPU direct sum (CudaDirectKde::unnormalized_eval ->
eval_kernel, include/CudaDirectKde.h:126-215, compiled unmodified for sm_100a into
oracle/_ref/libkde_ref_gpu.so) beside this project's pair sum on identical
inputs, both against the FP64 oracle.

The reference sums in plain FP32 (one running float per query, an expf and two
divisions per pair); the FP32-compensated sum here holds the reference's own
CPU-vs-GPU criterion approximately_equal(1e-6, 1e-8) (test/test_cukde2.cc:68-70)
at every query; the reference kernel is asserted only to plain-FP32 accuracy
(1e-4 relative: one running float over 30,000 terms)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from bbrcit_kde_b200.parity import error_stats

pytestmark = pytest.mark.gpu
SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                  "libkde_ref_gpu.so")


@pytest.mark.skipif(not os.path.exists(SO), reason="reference GPU harness not built")
@pytest.mark.parametrize("kind,h", [(W.GAUSS_PROD2D, (0.05, 0.08)), (W.GAUSS, (0.1, 0.1)),
                                    (W.EPAN, (0.3, 0.3))])
def test_reference_gpu_kernel_and_ours_against_fp64(ctx, oracle, kind, h):
    wl = W.config2(n=30_000, m=4_096)
    wn = wl.weights / wl.weights.sum()
    refs, qs = np.ascontiguousarray(wl.refs), np.ascontiguousarray(wl.queries)
    dp = C.POINTER(C.c_double)
    lib = C.CDLL(SO)
    lib.ref_gpu_direct.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int64, dp, dp, dp,
                                   C.c_int64, dp, C.c_int, C.c_int, dp, dp]
    ref_out, ms = np.empty(len(qs)), C.c_double(0.0)
    wn_c = np.ascontiguousarray(wn)
    rc = lib.ref_gpu_direct(kind, h[0], h[1], len(refs), refs.ctypes.data_as(dp),
                            wn_c.ctypes.data_as(dp), None, len(qs), qs.ctypes.data_as(dp), 128,
                            1, ref_out.ctypes.data_as(dp), C.byref(ms))
    assert rc == 0
    ctx.upload(bk.REFERENCE, refs, mass=wn, weight=wn)
    ctx.upload(bk.QUERY, qs)
    ours = ctx.eval_all(bk.kernel_desc(kind, 2, h))
    want = oracle.direct(kind, 2, h, refs, wn, qs)
    s_ours = error_stats(ours, want, 1e-6, 1e-8)
    s_ref = error_stats(ref_out, want, 1e-4, 1e-8)
    assert s_ours["pass_rate"] == 1.0, s_ours
    assert s_ref["pass_rate"] == 1.0, s_ref
