"""Factored grid sums on the tcgen05 tensor cores (k_pair_sum_culled_sep_tc).

The 32 x 32-tile factored sum can run its accumulation as TF32 MMAs with every
kernel factor split into two TF32 terms (bbkde_grid_config.tensor_cores). The
split keeps 22 of a factor's 24 bits and the tensor core accumulates 32
references per FP32 partial, so against FP64 each point is within about 1e-6
relative (measured on the device: at most 6e-7 per 32-reference partial).

Tolerances:
  against the FP32C direct path -- every point within rel 3e-6 (the direct
      path's 1e-6 bar plus the split's error budget), abs 1e-8 as the grid tests;
  against the FP32-pipe factored form of the same culled sum -- rel 3e-6;
  repeated calls -- bitwise equal (the MMA chain has a fixed order).
"""
from __future__ import annotations

import numpy as np
import pytest

import bbrcit_kde_b200 as bk
from bbrcit_kde_b200 import workloads as W
from tests.helpers import assert_parity

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TC_REL = 3e-6
GRID = (250, 190, -3.0, 3.0, -2.5, 2.5)     # partial edge tiles on both axes


def _grid_points(grid):
    nx, ny, x0, x1, y0, y1 = grid
    return W.grid_2d(x0, x1, nx, y0, y1, ny)


def _grid_eval(ctx, desc, grid, **kw):
    out = torch.empty(grid[0] * grid[1], dtype=torch.float64, device="cuda")
    st = ctx.eval_grid(desc, grid, out.data_ptr(), **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy(), st


def _direct_on_grid(ctx, desc, grid):
    ctx.upload(bk.QUERY, _grid_points(grid))
    return ctx.eval_all(desc)


def _adaptive_refs(ctx, n=60_000):
    refs = W.config5_refs(n)
    ctx.upload(bk.REFERENCE, refs, mass=np.full(n, 1.0 / n), weight=np.full(n, 1.0 / n))
    desc = bk.kernel_desc(W.GAUSS, 2, (0.08, 0.08))
    ctx.adapt_density(desc, 0.5, outputs=False)
    return desc


@pytest.mark.parametrize("kind,h", [(W.GAUSS, None), (W.GAUSS_PROD2D, (0.05, 0.09)),
                                    (W.EPAN_PROD2D, (0.2, 0.15))])
def test_tensor_core_tiles_match_direct_and_fp32_pipe(ctx, kind, h):
    """Every separable kernel on a ragged grid: the tensor-core form against the
    direct path and against the FP32-pipe form of the same culled sum."""
    if kind == W.GAUSS:
        desc = _adaptive_refs(ctx)
    else:
        n = 60_000
        refs = W.config5_refs(n)
        abw = W.SplitMix64(404).uniform(n, 0.5, 2.0)
        ctx.upload(bk.REFERENCE, refs, mass=np.full(n, 1.0 / n) * abw ** -2, abw=abw)
        desc = bk.kernel_desc(kind, 2, h)
    want = _direct_on_grid(ctx, desc, GRID)
    tc, st = _grid_eval(ctx, desc, GRID, mode=bk.GRID_EXACT, tile=32, tensor_cores=2)
    s = assert_parity(tc, want, TC_REL, 1e-8, what=f"kind {kind} tensor cores")
    assert st.max_bound_ratio <= 1e-7 and st.exact_points == GRID[0] * GRID[1]
    fp32, _ = _grid_eval(ctx, desc, GRID, mode=bk.GRID_EXACT, tile=32, tensor_cores=1)
    assert_parity(tc, fp32, TC_REL, 1e-8, what=f"kind {kind} tensor cores vs FP32 pipe")
    again, _ = _grid_eval(ctx, desc, GRID, mode=bk.GRID_EXACT, tile=32, tensor_cores=2)
    assert np.array_equal(tc, again)
    assert s["max_rel_sig"] <= TC_REL, s


def test_tensor_core_tiles_long_list_and_automatic_choice(ctx):
    """The automatic setting takes the tensor cores for every culled tile-32 sum at
    tolerances of 1e-5 and above: 128-thread blocks for lists of at least 16
    waves (a ragged 3200 x 3100 grid, 9,700 tiles, in the most-expensive-first
    launch order), 256-thread blocks for shorter ones (a 1,024-tile list). Both
    are bitwise the forced result and match the direct sum and the FP32-pipe
    form; at 1e-7 every list stays on the FP32 pipe (bitwise the forced
    FP32-pipe result)."""
    desc = _adaptive_refs(ctx)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for grid, what in (((3200, 3100, -4.0, 4.0, -4.0, 4.0), "9,700 tiles"),
                       ((1000, 990, -4.0, 4.0, -4.0, 4.0), "1,024 tiles")):
        tiles = ((grid[0] + 31) // 32) * ((grid[1] + 31) // 32)
        assert (tiles >= 16 * 4 * sms) == (tiles == 9700)
        want = _direct_on_grid(ctx, desc, grid)
        auto5, st = _grid_eval(ctx, desc, grid, mode=bk.GRID_EXACT, tile=32, cull_rel=1e-5)
        forced5, _ = _grid_eval(ctx, desc, grid, mode=bk.GRID_EXACT, tile=32, cull_rel=1e-5,
                                tensor_cores=2)
        assert np.array_equal(auto5, forced5)
        assert_parity(auto5, want, 1e-5 + TC_REL, 1e-8, what=f"{what}, 1e-5, tensor cores")
        assert st.max_bound_ratio <= 1e-5
        fp5, _ = _grid_eval(ctx, desc, grid, mode=bk.GRID_EXACT, tile=32, cull_rel=1e-5,
                            tensor_cores=1)
        assert_parity(auto5, fp5, TC_REL, 1e-8, what=f"{what}, tensor cores vs FP32 pipe")
        auto7, _ = _grid_eval(ctx, desc, grid, mode=bk.GRID_EXACT, tile=32, cull_rel=1e-7)
        fp7, _ = _grid_eval(ctx, desc, grid, mode=bk.GRID_EXACT, tile=32, cull_rel=1e-7,
                            tensor_cores=1)
        assert np.array_equal(auto7, fp7)
        assert_parity(auto7, want, 1e-6 + 1e-7, 1e-8, what=f"{what}, 1e-7, FP32 pipe")


def test_tensor_cores_setting_is_checked(ctx):
    desc = _adaptive_refs(ctx, n=5_000)
    for bad in (-1, 3):
        with pytest.raises(bk.InvalidArgument):
            _grid_eval(ctx, desc, (64, 64, -1.0, 1.0, -1.0, 1.0), mode=bk.GRID_EXACT, tile=32,
                       tensor_cores=bad)
