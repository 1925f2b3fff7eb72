"""The allocation-free entry point bbkde_eval_noalloc, through the C ABI.

It serves callers that cannot call cudaMalloc (a host framework that owns every
device allocation through its own pool, or code that must run when allocation is
forbidden or memory is exhausted): they pass device buffers for inputs and
output, and the scratch comes from one fixed array in the library's device
image. This file is collected last so that, when it fails, a run stopping at the
first failure has already run every other test; it also passes on its own.
"""
from __future__ import annotations

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from bbrcit_kde_b200.parity import error_stats

pytestmark = pytest.mark.gpu


def _problem(seed, n, m, dim):
    rng = W.SplitMix64(seed)
    refs = W.f32(rng.normal(n * dim).reshape(n, dim))
    q = W.f32(rng.uniform(m * dim, -3, 3).reshape(m, dim))
    mass = rng.uniform(n, 0.5, 2.0) / n
    abw = rng.uniform(n, 0.5, 2.0)
    return refs, q, mass, abw


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def test_noalloc_matches_context_path_twice(ctx):
    torch = pytest.importorskip("torch")
    cases = [(W.GAUSS_PROD2D, 2, (0.05, 0.08), 20011, 30007),
             (W.EPAN, 2, (0.3, 0.3), 7001, 12289),
             (W.GAUSS, 1, (0.02, 0.02), 50000, 9000)]
    stream = torch.cuda.current_stream().cuda_stream
    free_after = []
    for call, (kind, dim, h, n, m) in enumerate(cases):
        refs, q, mass, abw = _problem(500 + call, n, m, dim)
        desc = bk.kernel_desc(kind, dim, h)
        ctx.upload(bk.REFERENCE, refs, mass=mass, abw=abw)
        ctx.upload(bk.QUERY, q)
        want = ctx.eval_all(desc, precision=bk.FP32C)
        rx, rm, ra, qx = _dev(torch, refs[:, 0]), _dev(torch, mass), _dev(torch, abw), \
            _dev(torch, q[:, 0])
        ry = _dev(torch, refs[:, 1]) if dim == 2 else None
        qy = _dev(torch, q[:, 1]) if dim == 2 else None
        out = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc, msg = bk.eval_noalloc(desc, n, rx.data_ptr(), ry.data_ptr() if ry is not None else None,
                                  rm.data_ptr(), ra.data_ptr(), m, qx.data_ptr(),
                                  qy.data_ptr() if qy is not None else None, out.data_ptr(),
                                  True, stream)
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        assert rc == bk.OK, msg
        assert free_after[-1] == free0, "the allocation-free call changed free device memory"
        got = out.cpu().numpy()
        s = error_stats(got, want, 1e-6, 1e-8)
        assert s["pass_rate"] == 1.0, (call, s)
        np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-12)


def test_noalloc_rejects_oversize_and_bad_arguments():
    torch = pytest.importorskip("torch")
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    desc = bk.kernel_desc(W.GAUSS, 2, (0.1,))
    p = x.data_ptr()
    # 8,000,000 references need 128 MB of records: rejected before any launch.
    rc, msg = bk.eval_noalloc(desc, 8_000_000, p, p, p, None, 4, p, p, p)
    assert rc == bk.OUT_OF_RANGE and "scratch" in msg
    rc, msg = bk.eval_noalloc(desc, 4, p, p, p, None, 20_000_000, p, p, p)
    assert rc == bk.OUT_OF_RANGE and "scratch" in msg
    rc, msg = bk.eval_noalloc(desc, 4, p, None, p, None, 4, p, p, p)   # 2-D needs ref_y
    assert rc == bk.INVALID_ARGUMENT
    rc, msg = bk.eval_noalloc(bk.kernel_desc(W.GAUSS, 2, (0.0,)), 4, p, p, p, None, 4, p, p, p)
    assert rc == bk.INVALID_ARGUMENT
    rc, msg = bk.eval_noalloc(desc, 4, p, p, p, None, 0, p, p, p)     # nothing to do
    assert rc == bk.OK
    # Counts whose byte sizes would wrap a 64-bit product are rejected on the host
    # before any arithmetic on them, and before any launch.
    for n_ref, n_query in ((2**60 + 5, 4), (4, 2**60 + 5), (2**62, 2**62)):
        rc, msg = bk.eval_noalloc(desc, n_ref, p, p, p, None, n_query, p, p, p)
        assert rc == bk.OUT_OF_RANGE and "scratch" in msg, (n_ref, n_query, msg)


def test_noalloc_at_documented_capacity(ctx):
    """1,000,000 references x 1,000,000 2-D queries with a product kernel (20 B per
    reference) and no bandwidth column: the largest problem the header promises.
    Here the scratch, not the launch planner, limits the segment count, and the
    query columns and partials sit at the end of the array."""
    torch = pytest.importorskip("torch")
    n = m = 1_000_000
    refs, q, mass, _ = _problem(777, n, m, 2)
    desc = bk.kernel_desc(W.GAUSS_PROD2D, 2, (0.05, 0.07))
    ctx.upload(bk.REFERENCE, refs, mass=mass)
    ctx.upload(bk.QUERY, q)
    want = ctx.eval_all(desc, precision=bk.FP32C)
    cols = [_dev(torch, c) for c in (refs[:, 0], refs[:, 1], mass, q[:, 0], q[:, 1])]
    out = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rx, ry, rm, qx, qy = (c.data_ptr() for c in cols)
    rc, msg = bk.eval_noalloc(desc, n, rx, ry, rm, None, m, qx, qy, out.data_ptr(), True,
                              stream)
    torch.cuda.synchronize()
    assert rc == bk.OK, msg
    assert torch.cuda.mem_get_info()[0] == free0
    got = out.cpu().numpy()
    s = error_stats(got, want, 1e-6, 1e-8)
    assert s["pass_rate"] == 1.0, s
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-12)


_FIRST_CALL = r"""
import sys
sys.path.insert(0, sys.argv[1])
import numpy as np
import torch
import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W

torch.cuda.init()
rng = W.SplitMix64(4242)
n, m = 30011, 20011
refs = W.f32(rng.normal(2 * n).reshape(n, 2))
q = W.f32(rng.uniform(2 * m, -3, 3).reshape(m, 2))
mass = rng.uniform(n, 0.5, 2.0) / n
abw = rng.uniform(n, 0.5, 2.0)
dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
cols = [dev(c) for c in (refs[:, 0], refs[:, 1], mass, abw, q[:, 0], q[:, 1])]
rx, ry, rm, ra, qx, qy = (c.data_ptr() for c in cols)
out = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
desc = bk.kernel_desc(W.GAUSS_PROD2D, 2, (0.05, 0.08))
stream = torch.cuda.current_stream().cuda_stream
# the library's first call in this process: no queries, it only places the array
rc, msg = bk.eval_noalloc(desc, n, rx, ry, rm, ra, 0, qx, qy, out.data_ptr(), True, stream)
assert rc == bk.OK, msg
torch.cuda.synchronize()
free0 = torch.cuda.mem_get_info()[0]
got = []
for _ in range(2):
    out.fill_(float("nan"))
    torch.cuda.synchronize()
    rc, msg = bk.eval_noalloc(desc, n, rx, ry, rm, ra, m, qx, qy, out.data_ptr(), True, stream)
    torch.cuda.synchronize()
    assert rc == bk.OK, msg
    assert torch.cuda.mem_get_info()[0] == free0, "free device memory changed"
    got.append(out.cpu().numpy())
with bk.Context(0) as ctx:
    ctx.upload(bk.REFERENCE, refs, mass=mass, abw=abw)
    ctx.upload(bk.QUERY, q)
    want = ctx.eval_all(desc, precision=bk.FP32C)
for g in got:
    np.testing.assert_allclose(g, want, rtol=1e-6, atol=1e-12)
np.testing.assert_array_equal(got[0], got[1])
print("FIRST_CALL_OK")
"""


def test_noalloc_as_first_library_call_in_a_fresh_process():
    """A process whose first use of the library is bbkde_eval_noalloc: the
    n_query = 0 set-up call loads the array, after which evaluations leave free
    device memory unchanged and match the context path."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL, root], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0 and "FIRST_CALL_OK" in r.stdout, r.stdout + r.stderr
