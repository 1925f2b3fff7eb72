"""Host-side checks of the tensor-core factored grid sum (csrc/kde_culled_sep_tc.cuh).

1. The two-term TF32 split of a kernel factor (tf32_split2): with c = 8193 v,
   hi = c - (c - v) and lo = v - hi. numpy float32 arithmetic rounds to nearest
   like the device's FP32 pipe (the kernel writes a - b as fma(b, -1, a), which
   rounds once, as a subtraction). The tensor core reads a TF32 operand from an
   FP32 word's sign, exponent and top 10 mantissa bits, modelled here by clearing
   the low 13 bits of lo. Checked: hi carries at most 11 significant bits (an
   exact TF32 operand), lo = v - hi exactly, and v - hi - tf32(lo) is below
   2^-21 |v| over factors from 1e-30 to 1e4.
2. The index mappings of both block shapes (128 and 256 threads). A's row 16 q + 8 p + i holds part
   p (hi, lo) of tile row 8 q + i, and B's row c + 32 p holds part p of column c.
   An M = 64 accumulator row m sits in TMEM lane (m / 16) * 32 + m % 16. A
   tcgen05.ld 16x256b.x(512 / NT) at column c0 gives thread t register 4 j + e =
   (lane t / 4, column c0 + 8 j + 2 (t % 4) + e) and register 4 j + 2 + e = (lane
   8 + t / 4, the same column) of its warp's lane quarter. With 256 threads, warps
   w and w + 4 share quarter w % 4 and read column halves w / 4.
   Checked: the four registers the fold adds for each of a thread's points are
   the four quadrant products of that point's own row and column, and the
   threads cover the 32 x 32 tile once. The factor-making threads write every
   (operand row, reference quad) of both operands once, and 128 contiguous bytes
   per 8 lanes.
"""
from __future__ import annotations

import numpy as np
import pytest

f32 = np.float32


def _veltkamp11(v):
    c = (v * f32(8193.0)).astype(f32)
    t = (c - v).astype(f32)
    return (c - t).astype(f32)


def _tf32_read(x):
    """What the tensor core takes from an FP32 word: the low 13 bits dropped."""
    return (x.astype(f32).view(np.uint32) & np.uint32(0xFFFFE000)).view(f32)


def _split(v):
    hi = _veltkamp11(v)
    lo = (v - hi).astype(f32)
    return hi, lo


def _significant_bits(x):
    """Bits from the leading one to the last one of the float32 significand."""
    b = x.astype(f32).view(np.uint32)
    mant = (b & np.uint32(0x7FFFFF)) | np.uint32(0x800000)
    tz = np.zeros(b.shape, dtype=np.int64)
    m = mant.astype(np.int64)
    for _ in range(24):
        odd = (m & 1) == 1
        tz = np.where(odd, tz, tz + 1)
        m = np.where(odd, m, m >> 1)
    return np.where(x == 0, 0, 24 - tz)


def test_tf32_split_terms_are_exact_and_remainder_bounded():
    rng = np.random.default_rng(7)
    v = np.concatenate([
        f32(10.0) ** rng.uniform(-30, 4, 200_000).astype(f32),
        rng.uniform(0, 1, 100_000).astype(f32),
        np.array([1.0, 0.5, 2 ** -20, 1 - 2 ** -24, 3.0, 1e-38], dtype=f32),
    ]).astype(f32)
    v = v[np.isfinite(v) & (v > 0) & (v >= f32(1e-30))]
    hi, lo = _split(v)
    assert _significant_bits(hi).max() <= 11
    assert np.array_equal(hi.astype(np.float64) + lo.astype(np.float64), v.astype(np.float64))
    assert np.all(np.abs(lo.astype(np.float64)) <= 2.0 ** -11 * v.astype(np.float64))
    rest = v.astype(np.float64) - hi.astype(np.float64) - _tf32_read(lo).astype(np.float64)
    assert np.all(np.abs(rest) < 2.0 ** -21 * v.astype(np.float64))
    # hi alone leaves up to 2^-11 of v
    assert np.max(np.abs(v.astype(np.float64) - hi) / v) > 2.0 ** -14


def test_quadrant_product_of_split_factors():
    """Y X^T from the four quadrants of [Y_hi; Y_lo] [X_hi; X_lo]^T, as the tensor
    core reads the operands, against FP64 of the FP32 factors, with exact (FP64)
    products: what is left is the split, below 2^-20 of each product."""
    rng = np.random.default_rng(11)
    y = (2.0 ** rng.uniform(-20, 0, (32, 32))).astype(f32)
    x = (2.0 ** rng.uniform(-20, 0, (32, 32))).astype(f32)
    yh, yl = _split(y)
    xh, xl = _split(x)
    a = _tf32_read(np.concatenate([yh, yl])).astype(np.float64)
    b = _tf32_read(np.concatenate([xh, xl])).astype(np.float64)
    assert np.array_equal(_tf32_read(yh), yh)
    d = a @ b.T
    got = d[32:, :32] + d[:32, 32:] + d[32:, 32:] + d[:32, :32]
    want = y.astype(np.float64) @ x.astype(np.float64).T
    assert np.max(np.abs(got - want) / want) <= 2.0 ** -20


@pytest.mark.parametrize("nt", [128, 256])
def test_operand_rows_and_fragment_give_each_point_its_quadrants(nt):
    # accumulator entry (m, n) tagged by the product it holds
    def a_row(tile_row, part):
        return 16 * (tile_row // 8) + 8 * part + tile_row % 8

    tag = {}
    for r in range(32):
        for p in range(2):
            for c in range(32):
                for q in range(2):
                    tag[(a_row(r, p), c + 32 * q)] = (r, c, p, q)
    assert len(tag) == 64 * 64
    lane_of_row = {m: (m // 16) * 32 + m % 16 for m in range(64)}
    row_of_lane = {ln: m for m, ln in lane_of_row.items()}

    pp = 512 // nt     # point pairs per thread: 4 at 128 threads, 2 at 256

    def ld(lane_base, col_base, t):
        """16x256b.x{pp}: register -> (TMEM lane, column) for thread t."""
        regs = {}
        for j in range(pp):
            for e in range(2):
                col = col_base + 8 * j + 2 * (t % 4) + e
                regs[4 * j + e] = (lane_base + t // 4, col)
                regs[4 * j + 2 + e] = (lane_base + 8 + t // 4, col)
        return regs

    covered = np.zeros((32, 32), dtype=int)
    for warp in range(nt // 32):
        lq, ch = warp % 4, warp // 4
        for t in range(32):
            v = ld(32 * lq, 8 * pp * ch, t)          # X_hi columns of this warp
            w = ld(32 * lq, 32 + 8 * pp * ch, t)     # X_lo columns
            prow = 8 * lq + t // 4
            for k in range(2 * pp):
                j, e = k // 2, k % 2
                pcol = 8 * (pp * ch + j) + 2 * (t % 4) + e
                # the fold adds lo.hi, hi.lo, lo.lo, hi.hi
                got = set()
                for lane, col in (v[4 * j + 2 + e], w[4 * j + e], w[4 * j + 2 + e], v[4 * j + e]):
                    r, c, p, q = tag[(row_of_lane[lane], col)]
                    assert (r, c) == (prow, pcol)
                    got.add((p, q))
                assert got == {(1, 0), (0, 1), (1, 1), (0, 0)}
                covered[prow, pcol] += 1
    assert np.all(covered == 1)


@pytest.mark.parametrize("nt", [128, 256])
def test_factor_threads_cover_both_operands_once(nt):
    """kg = (t / 16) % 8, half = (t / 8) % 2, r8 = t % 8, rs = t / 128, rows i =
    PP rs + i', i' < PP = 512 / NT: every (operand row, reference quad) is written
    once, and each 8-lane group writes one 8-row core matrix (128 contiguous
    bytes)."""
    pp = 512 // nt
    def off(m, k):
        return (k // 4) * 1024 + (m // 8) * 128 + (m % 8) * 16 + (k % 4) * 4

    seen = {}
    for t in range(nt):
        kg, half, r8, rs = (t // 16) % 8, (t // 8) % 2, t % 8, t // 128
        for i in range(pp * rs, pp * rs + pp):
            mh = r8 + 8 * i if half else 16 * i + r8
            ml = 32 + r8 + 8 * i if half else 16 * i + 8 + r8
            for m in (mh, ml):
                key = (half, m, kg)
                assert key not in seen
                seen[key] = t
                assert off(m, 4 * kg) + 16 <= 8192
    assert len(seen) == 2 * 64 * 8
    for t0 in range(0, nt, 8):
        for i_sel in range(pp):
            offs = []
            for t in range(t0, t0 + 8):
                kg, half, r8, rs = (t // 16) % 8, (t // 8) % 2, t % 8, t // 128
                i = pp * rs + i_sel
                m = r8 + 8 * i if half else 16 * i + r8
                offs.append(off(m, 4 * kg))
            assert sorted(offs) == list(range(min(offs), min(offs) + 128, 16))
