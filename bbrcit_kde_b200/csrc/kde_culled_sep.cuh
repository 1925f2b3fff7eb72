// Culled exact sum on grid tiles for the separable kernels.
//
// The Gaussian kernels (isotropic and product) and the Epanechnikov product
// kernel factor over the axes: U(q - r) = u_x(q_x - r_x) * u_y(q_y - r_y). On a
// T x T tile of grid points the T columns share their x and the T rows their y,
// so per reference the block evaluates u_x at the T columns and m * u_y at the T
// rows -- 2T kernel factors (2T MUFU.EX2 for the Gaussians) instead of T^2 --
// and every point then accumulates one product. The Gaussian sum leaves the MUFU
// bound (16 pairs per clock per SM): 2T exponentials and T^2 multiply-adds per
// reference, ~T^2/2T = T/2 times fewer exponentials than pairs.
//
// Culling is k_pair_sum_culled's (kde_culled.cuh): Morton-sorted 256-reference
// tiles scanned two levels deep (tile groups first), near field within 2^-cut of
// the largest tile bound, far field against per-slot thresholds (slot k = the
// k-th strip of T/8 rows), every skipped unit booked in the per-slot bound
// (skipped part < rel * S_k / 2). One difference in the flush rule: a tile whose
// largest pair exponent is below -128 is skipped here too, but a product of two
// factors may be a denormal instead of the direct path's flushed zero, i.e. such
// a tile would add less than 2^-126 * mass per pair.
//
// Per summed tile: the 256 records are staged in shared memory by coalesced
// read-only loads (coordinates negated, x and y columns side by side); then,
// per sub-chunk of SUB references, thread w of each 2T-thread team computes the
// factor of column w (w < T) or of row w - T for two references at a time with
// packed f32x2 arithmetic, stored as (even, odd) reference pairs; the points
// then accumulate two partial sums (even and odd references) with FFMA2.
//
// Layout: block = T*T/8 threads in two splits of T*T/16 lanes; split sp takes
// the reference pairs p with p % 2 == sp, and its lane (rg, cg) owns the 4 x 4
// points of rows {2rg, 2rg + 1, T/2 + 2rg, T/2 + 2rg + 1} and the same columns
// with cg: per reference pair 4 128-bit loads of factors feed 16 FFMA2. For
// T = 16 both splits share a warp: odd factor rows are stored with the column
// index XOR 8, so that the splits' loads fall on different banks.
//
// Software pipeline: the factors of sub-chunk s + 1 are computed in the same
// loop body as the accumulation of sub-chunk s (double-buffered), so that the
// MUFU/FMA chains of the one and the loads and FFMA2 of the other overlap
// within every warp. Summation: FP32
// partial sums of kChunk references (two interleaved halves) folded into
// per-point Kahan accumulators, tiles in ascending sorted order, near field
// before far field; the two splits are added in FP64 at the end (split 0 +
// split 1) -- deterministic.
#pragma once

#include <cooperative_groups.h>
#include <cstdint>
#include <cuda_runtime.h>

#include "kde_culled.cuh"

namespace bbkde {

__host__ __device__ constexpr bool op_separable(int op) {
  return op == OP_GAUSS_ISO || op == OP_GAUSS_PROD || op == OP_EPAN_PROD;
}

// Split tiles (S > 1, launched as clusters of S blocks per tile): for short tile
// lists, where one block per tile would leave most SMs idle while the densest
// tiles finish, block `part` of a tile's cluster sums every S-th batch of tile
// groups. Every part scans all groups for the largest bound (the same near/far
// split), the parts exchange their near-field sums through distributed shared
// memory so that all of them use the thresholds of the total near-field sum, and
// part 0 adds the parts' point sums in rank order. The skipped units of the
// parts are disjoint subsets of one tile's units, so their bounds add up to the
// single-block bound (reported by part 0 from the parts' sums).
template <int OP, int T, int S = 1>
__global__ void __launch_bounds__(T *T / 8, T == 32 ? 4 : 16)
    k_pair_sum_culled_sep(CullArgs a) {
  static_assert(T == 16 || T == 32, "tile edge");
  constexpr int BLOCK = T * T / 8;
  constexpr int NW = BLOCK / 32;
  constexpr int LPS = T * T / 16;      // lanes per split (16 points each)
  constexpr int CG = T / 4;            // column groups of a split
  constexpr int NS = 8;                // slots: strips of T / 8 rows
  constexpr int SPR = T / NS;          // rows per slot
  constexpr int SUB = T == 16 ? 32 : 64;   // references per factor sub-chunk
  constexpr int NSUB = kRefTile / SUB;
  constexpr int FROWS = SUB / 2;       // reference pairs per sub-chunk
  constexpr int FBUF = 2 * FROWS * T;  // factor pairs per buffer (x rows, then y rows)
  constexpr int STG = kRefTile + 4;    // staged column stride (x and y on different banks)
  constexpr bool kGauss = op_gauss(OP);
  constexpr bool kExt = op_has_extra(OP);
  static_assert(BLOCK == 2 * LPS, "two splits");
  static_assert(kChunk == 32, "partials of the pair form's chunk");
  static_assert(kRefTile % SUB == 0 && FROWS % (kChunk / 2) == 0, "shape");
  static_assert(FBUF >= T * T, "exchange area: two T x T double arrays");
  static_assert(S == 1 || S == 2 || S == 4 || S == 8, "cluster size");
  __shared__ __align__(16) float s_c[2 * STG];     // -x | -y of the staged references
  __shared__ __align__(16) float s_s[2 * STG];     // x scale | y scale
  __shared__ __align__(16) float s_m[2 * STG];     // 1 | mass
  // Two buffers of u_x rows ([pair][column], (even, odd)) then m u_y rows;
  // reused to hand split 1's sums to split 0.
  __shared__ __align__(16) float2 s_fac[2 * FBUF];
  __shared__ float s_qx[T], s_qy[T];
  __shared__ int s_list[cull_list_len(BLOCK)];
  __shared__ int s_glist[cull_groups_per_batch(BLOCK)];
  __shared__ int s_wc[NW];
  __shared__ float s_box[NS][4];
  __shared__ float s_th[NS];
  __shared__ unsigned s_min[NS];       // bits of the slot's smallest near-field sum (>= 0)
  __shared__ float s_red[NW];
  __shared__ double s_d[NS][NW];
  __shared__ float s_near[S > 1 ? T * T : 1];   // this part's near-field point sums
  __shared__ double s_b[NS];                      // this part's skipped bound per slot
  __shared__ int s_summed;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int sp = tid / LPS, rg = (tid % LPS) / CG, cg = (tid % LPS) % CG;
  const CullQueries &q = a.q;
  const int part = S > 1 ? (int)(blockIdx.x % S) : 0;
  const int64_t tile_slot = blockIdx.x / S;
  const int t = q.tile_list[tile_slot];
  const int64_t i0 = (int64_t)(t % q.ntx) * T, j0 = (int64_t)(t / q.ntx) * T;
  if (tid < T) {
    s_qx[tid] = grid_coord(q.gx0, q.gdx, i0 + tid);
    s_qy[tid] = grid_coord(q.gy0, q.gdy, j0 + tid);
  }
  for (int i = tid; i < kRefTile; i += BLOCK) s_m[i] = 1.0f;
  if (tid < NS) {
    // slot tid: rows j0 + tid T/8 .. + T/8 - 1 and all columns, inside the grid
    const int64_t jlo = j0 + (int64_t)tid * SPR;
    const int64_t jhi = (jlo + SPR < q.gny ? jlo + SPR : q.gny) - 1;
    const int64_t ihi = (i0 + T < q.gnx ? i0 + T : q.gnx) - 1;
    if (jlo < q.gny) {
      s_box[tid][0] = grid_coord(q.gx0, q.gdx, i0);
      s_box[tid][1] = grid_coord(q.gx0, q.gdx, ihi);
      s_box[tid][2] = grid_coord(q.gy0, q.gdy, jlo);
      s_box[tid][3] = grid_coord(q.gy0, q.gdy, jhi);
    } else {
      s_box[tid][0] = 3e38f; s_box[tid][1] = -3e38f;
      s_box[tid][2] = 3e38f; s_box[tid][3] = -3e38f;
    }
    s_min[tid] = 0x7f800000u;   // +inf
  }
  __syncthreads();
  float qx0 = 3e38f, qx1 = -3e38f, qy0 = 3e38f, qy1 = -3e38f;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    qx0 = fminf(qx0, s_box[k][0]); qx1 = fmaxf(qx1, s_box[k][1]);
    qy0 = fminf(qy0, s_box[k][2]); qy1 = fmaxf(qy1, s_box[k][3]);
  }
  // The lane's rows and columns: k = 0, 1 -> 2g + k; k = 2, 3 -> T/2 + 2g + k - 2.
  auto own = [](int g, int k) { return (k < 2 ? 0 : T / 2) + 2 * g + (k & 1); };
  // Kahan accumulators of the 16 points, two points (k = 2i, 2i + 1: the same
  // row, adjacent columns) per packed pair.
  float2 sum[8], comp[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) { sum[k] = f2(0.f); comp[k] = f2(0.f); }
  auto point_sum = [&](int k) -> float {
    return (k & 1) ? sum[k >> 1].y - comp[k >> 1].y : sum[k >> 1].x - comp[k >> 1].x;
  };
  auto point_sum_d = [&](int k) -> double {
    return (k & 1) ? (double)sum[k >> 1].y - (double)comp[k >> 1].y
                   : (double)sum[k >> 1].x - (double)comp[k >> 1].x;
  };

  // This thread's factor: column w or row w - T of team ft.
  // Factor teams of T threads: thread f of a team computes columns (f < T/2) or
  // rows (f >= T/2) 2 (f mod T/2) and 2 (f mod T/2) + 1, two references at a
  // time, so that each broadcast load of a reference pair's record feeds two
  // factors; team ft takes the pairs ft, ft + NTM, ... of a sub-chunk.
  constexpr int NTM = BLOCK / T;       // factor teams: 4 at T = 32, 2 at T = 16
  static_assert(FROWS / NTM == 8, "eight factor calls per sub-chunk and lane");
  const int fl = tid % T, ft = tid / T;
  const bool fx = fl < T / 2;
  const int fcol = 2 * (fl % (T / 2));
  const float fq = fx ? s_qx[fcol] : s_qy[fcol];
  const float fq1 = fx ? s_qx[fcol + 1] : s_qy[fcol + 1];
  const int foff = fx ? 0 : STG;
  float2 *const fbase = s_fac + (fx ? 0 : FROWS * T);
  // Column swizzle of factor row p (see the layout note).
  auto swz = [](int p) { return T == 16 ? (p & 1) << 3 : 0; };

  // Scan 1 (Gaussians): largest tile bound over the block's box.
  float e_max = -INFINITY;
  if (kGauss)
    e_max = cull_max<BLOCK>(a, s_red, [&](const RefTile &rt) {
      return rt.lm + tile_peak<OP, 2>(rt, qx0, qx1, qy0, qy1);
    });
  const float t_a = e_max - a.cut;

  float skipped[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) skipped[k] = 0.f;
  int summed = 0;

  // Is tile (or group) rt needed? (as in k_pair_sum_culled)
  auto needed = [&](const RefTile &rt, int phase, bool group) -> bool {
    if (!kGauss) {
      bool need = false;
#pragma unroll
      for (int k = 0; k < NS; ++k)
        need |= tile_peak<OP, 2>(rt, s_box[k][0], s_box[k][1], s_box[k][2], s_box[k][3]) > 0.f;
      return need;
    }
    const float pb = tile_peak<OP, 2>(rt, qx0, qx1, qy0, qy1);
    if (pb < kFlushExp) return false;
    const bool near = rt.lm + pb >= t_a;
    if (phase == 1) return near;
    if (near && !group) return false;
    bool need = false;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const float pk = tile_peak<OP, 2>(rt, s_box[k][0], s_box[k][1], s_box[k][2], s_box[k][3]);
      need |= pk >= kFlushExp && rt.lm + pk >= s_th[k];
    }
    if (!need) {
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const float pk = tile_peak<OP, 2>(rt, s_box[k][0], s_box[k][1], s_box[k][2], s_box[k][3]);
        if (pk >= kFlushExp) skipped[k] += ex2_approx(rt.lm + pk - s_th[k]);
      }
    }
    return need;
  };

  // Sum the references [t0, t1) of one tile into the points' accumulators.
  auto sum_tile = [&](int64_t t0, int64_t t1) {
    constexpr int PER = kRefTile / BLOCK;
    float4 rec[PER];
    float ext[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int64_t rr = t0 + u * BLOCK + tid;
      rec[u] = rr < t1 ? __ldg(a.refs + rr) : make_float4(0.f, 0.f, 0.f, 0.f);
      ext[u] = kExt ? (rr < t1 ? __ldg(a.extra + rr) : 0.f) : rec[u].w;
    }
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int i = u * BLOCK + tid;
      s_c[i] = -rec[u].x;
      s_c[STG + i] = -rec[u].y;
      s_s[i] = rec[u].w;
      s_s[STG + i] = ext[u];
      s_m[STG + i] = rec[u].z;
    }
    __syncthreads();
    // Factor pair p of sub-chunk sub (references sub + 2p, + 1) into buffer b.
    auto factor = [&](int b, int sub, int p) {
      const int j = foff + sub + 2 * p;
      const float2 c2 = *reinterpret_cast<const float2 *>(&s_c[j]);
      const float2 s2 = *reinterpret_cast<const float2 *>(&s_s[j]);
      const float2 m2 = *reinterpret_cast<const float2 *>(&s_m[j]);
      const float2 d = __fadd2_rn(f2(fq), c2);
      const float2 dd = __fmul2_rn(d, d);
      float2 u;
      if (kGauss) {
        const float2 e = __fmul2_rn(s2, dd);
        u = make_float2(ex2_approx(e.x), ex2_approx(e.y));
      } else {
        u = __ffma2_rn(s2, dd, f2(1.0f));
        u = make_float2(fmaxf(u.x, 0.f), fmaxf(u.y, 0.f));
      }
      {
        // the second column, the same reference pair; both stored as one 128-bit
        // record (columns fcol, fcol + 1 stay adjacent under the swizzle)
        const float2 d1 = __fadd2_rn(f2(fq1), c2);
        const float2 dd1 = __fmul2_rn(d1, d1);
        float2 u1;
        if (kGauss) {
          const float2 e1 = __fmul2_rn(s2, dd1);
          u1 = make_float2(ex2_approx(e1.x), ex2_approx(e1.y));
        } else {
          u1 = __ffma2_rn(s2, dd1, f2(1.0f));
          u1 = make_float2(fmaxf(u1.x, 0.f), fmaxf(u1.y, 0.f));
        }
        const float2 v0 = __fmul2_rn(m2, u), v1 = __fmul2_rn(m2, u1);
        *reinterpret_cast<float4 *>(&fbase[b * FBUF + p * T + (fcol ^ swz(p))]) =
            make_float4(v0.x, v0.y, v1.x, v1.y);
      }
    };
    // acc[4 kr + kc] (+)= y[kr] * x[kc] for factor pair p of buffer b.
    auto step = [&](int b, int p, float2 (&acc)[16], bool first) {
      const float2 *fx2 = s_fac + b * FBUF + p * T, *fy2 = fx2 + FROWS * T;
      const int w = swz(p);
      const float4 ya = *reinterpret_cast<const float4 *>(&fy2[(2 * rg) ^ w]);
      const float4 yb = *reinterpret_cast<const float4 *>(&fy2[(T / 2 + 2 * rg) ^ w]);
      const float4 xa = *reinterpret_cast<const float4 *>(&fx2[(2 * cg) ^ w]);
      const float4 xb = *reinterpret_cast<const float4 *>(&fx2[(T / 2 + 2 * cg) ^ w]);
      const float2 y[4] = {make_float2(ya.x, ya.y), make_float2(ya.z, ya.w),
                           make_float2(yb.x, yb.y), make_float2(yb.z, yb.w)};
      const float2 x[4] = {make_float2(xa.x, xa.y), make_float2(xa.z, xa.w),
                           make_float2(xb.x, xb.y), make_float2(xb.z, xb.w)};
#pragma unroll
      for (int kr = 0; kr < 4; ++kr)
#pragma unroll
        for (int kc = 0; kc < 4; ++kc)
          acc[4 * kr + kc] = first ? __fmul2_rn(y[kr], x[kc])
                                   : __ffma2_rn(y[kr], x[kc], acc[4 * kr + kc]);
    };
    for (int p = ft; p < FROWS; p += NTM) factor(0, 0, p);
    __syncthreads();
    // One FP32 partial per sub-chunk and split (16 references at T = 16, 32 at
    // T = 32: two interleaved halves, as the pair form's kChunk), then its Kahan
    // fold, two points per packed op (a - b as fma(b, -1, a): exact negation, one
    // rounding, as the scalar subtraction).
    for (int sb = 0; sb < NSUB; ++sb) {
      const int cur = sb & 1;
      const bool more = sb + 1 < NSUB;
      float2 acc[16];
#pragma unroll
      for (int ch = 0; ch < FROWS / 16; ++ch) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          if (more) {
            // eight calls per sub-chunk: every other step at T = 32 (two parts),
            // every step at T = 16
            if constexpr (T == 32) {
              if ((i & 1) == 0) factor(cur ^ 1, (sb + 1) * SUB, ft + (ch * 4 + i / 2) * NTM);
            } else {
              factor(cur ^ 1, (sb + 1) * SUB, ft + i * NTM);
            }
          }
          step(cur, ch * 16 + 2 * i + sp, acc, ch == 0 && i == 0);
        }
      }
      const float2 m1 = f2(-1.0f);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const float2 v = make_float2(acc[2 * k].x + acc[2 * k].y,
                                     acc[2 * k + 1].x + acc[2 * k + 1].y);
        const float2 y = __ffma2_rn(comp[k], m1, v);
        const float2 t2 = __fadd2_rn(sum[k], y);
        comp[k] = __ffma2_rn(y, m1, __ffma2_rn(sum[k], m1, t2));
        sum[k] = t2;
      }
      __syncthreads();
    }
  };

  auto sum_list = [&](int running) {
    for (int li = 0; li < running; ++li) {
      const int64_t t0 = (int64_t)s_list[li] * kRefTile;
      sum_tile(t0, t0 + kRefTile < a.n_ref ? t0 + kRefTile : a.n_ref);
    }
  };

  auto pass = [&](int phase) {
    summed += cull_pass<BLOCK>(
        a, s_list, s_glist, s_wc, [&](const RefTile &g) { return needed(g, phase, true); },
        [&](const RefTile &rt) { return needed(rt, phase, false); }, sum_list, part, S);
  };

  // Point k = 4 kr + kc of this lane: row own(rg, kr), column own(cg, kc).
  auto valid = [&](int k) {
    return i0 + own(cg, k & 3) < q.gnx && j0 + own(rg, k >> 2) < q.gny;
  };

  double smin_all = 0.0, ratio = 0.0;
  if (kGauss) {
    pass(1);   // near field
    // Split 1 hands its near-field sums to split 0 (the factor area is free
    // between passes); split 0 books the smallest per slot.
    float *const xf = reinterpret_cast<float *>(s_fac);
    if (sp == 1) {
#pragma unroll
      for (int k = 0; k < 16; ++k) xf[own(rg, k >> 2) * T + own(cg, k & 3)] = point_sum(k);
    }
    __syncthreads();
    if constexpr (S > 1) {
      if (sp == 0) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int idx = own(rg, k >> 2) * T + own(cg, k & 3);
          s_near[idx] = point_sum(k) + xf[idx];
        }
      }
      cooperative_groups::this_cluster().sync();
    }
    if (sp == 0) {
      float m0 = INFINITY, m1 = INFINITY;   // slots of rows k < 2 and k >= 2
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (!valid(k)) continue;
        const int idx = own(rg, k >> 2) * T + own(cg, k & 3);
        float tot;
        if constexpr (S > 1) {
          // the total near-field sum, parts added in rank order
          tot = 0.f;
          for (int r = 0; r < S; ++r)
            tot += cooperative_groups::this_cluster().map_shared_rank(s_near, r)[idx];
        } else {
          tot = point_sum(k) + xf[idx];
        }
        const float v = fmaxf(tot, 0.f);
        if ((k >> 2) < 2) m0 = fminf(m0, v);
        else m1 = fminf(m1, v);
      }
      if (m0 < INFINITY) atomicMin(&s_min[own(rg, 0) / SPR], __float_as_uint(m0));
      if (m1 < INFINITY) atomicMin(&s_min[own(rg, 2) / SPR], __float_as_uint(m1));
    }
    __syncthreads();
    if (tid < NS) {
      const double mk = (double)__uint_as_float(s_min[tid]);
      const double allow = fmax(a.rel * mk, a.abs_n);   // the pair form's allowance
      s_th[tid] = allow > 0.0 ? (float)(log2(allow) - log2((double)a.n_tiles)) - 1.0f
                              : -INFINITY;
    }
    __syncthreads();
    pass(2);   // far field, bound of the rest
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double sk = skipped[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sk += __shfl_xor_sync(0xffffffffu, sk, o);
      if (lane == 0) s_d[k][warp] = sk;
    }
    __syncthreads();
    if (tid < NS) {
      double b = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) b += s_d[tid][w];
      s_b[tid] = b;
    }
    __syncthreads();
    smin_all = INFINITY;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const double mk = (double)__uint_as_float(s_min[k]);
      smin_all = fmin(smin_all, mk);
      if (S == 1 && s_b[k] > 0.0)
        ratio = fmax(ratio, s_b[k] * exp2((double)s_th[k]) / fmax(a.rel * mk, a.abs_n));
    }
  } else {
    pass(0);
    if (tid < NS) s_b[tid] = 0.0;
  }
  // Split 1's sums to split 0, which adds split 0 + split 1.
  double *const xd = reinterpret_cast<double *>(s_fac);
  __syncthreads();
  if (sp == 1) {
#pragma unroll
    for (int k = 0; k < 16; ++k)
      xd[own(rg, k >> 2) * T + own(cg, k & 3)] = point_sum_d(k);
  }
  __syncthreads();
  if constexpr (S == 1) {
    if (tid == 0) {
      a.blk_bound[tile_slot] = ratio;
      a.blk_smin[tile_slot] = smin_all;
      a.blk_tiles[tile_slot] = summed;
    }
    if (sp == 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        if (!valid(k)) continue;
        const int row = own(rg, k >> 2), col = own(cg, k & 3);
        q.out[(j0 + row) * q.gnx + (i0 + col)] =
            q.scale * (point_sum_d(k) + xd[row * T + col]);
      }
    }
  } else {
    // This part's point sums beside split 1's; part 0 adds the parts in rank order.
    double *const xp = xd + T * T;
    if (sp == 0) {
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int idx = own(rg, k >> 2) * T + own(cg, k & 3);
        xp[idx] = point_sum_d(k) + xd[idx];
      }
    }
    if (tid == 0) s_summed = summed;
    auto cluster = cooperative_groups::this_cluster();
    cluster.sync();
    if (part == 0) {
      if (sp == 0) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          if (!valid(k)) continue;
          const int row = own(rg, k >> 2), col = own(cg, k & 3), idx = row * T + col;
          double v = 0.0;
          for (int r = 0; r < S; ++r) v += cluster.map_shared_rank(xp, r)[idx];
          q.out[(j0 + row) * q.gnx + (i0 + col)] = q.scale * v;
        }
      }
      if (tid == 0) {
        int tiles = 0;
        for (int r = 0; r < S; ++r) tiles += *cluster.map_shared_rank(&s_summed, r);
        if (kGauss) {
          for (int k = 0; k < NS; ++k) {
            double b = 0.0;
            for (int r = 0; r < S; ++r) b += cluster.map_shared_rank(s_b, r)[k];
            const double mk = (double)__uint_as_float(s_min[k]);
            if (b > 0.0)
              ratio = fmax(ratio, b * exp2((double)s_th[k]) / fmax(a.rel * mk, a.abs_n));
          }
        }
        a.blk_bound[tile_slot] = ratio;
        a.blk_smin[tile_slot] = smin_all;
        a.blk_tiles[tile_slot] = tiles;
      }
    }
    cluster.sync();   // the parts' shared memory stays valid until part 0 has read it
  }
}

// Launch order of a long factored tile list, most expensive first (so that the
// last wave is not left to the densest tiles): key[w] = ~(the number of
// reference groups whose bound over tile tile_list[w]'s box lies within `reach`
// (log2 units) of the largest such bound; for the Epanechnikov product, groups
// whose support meets the box) -- about the groups the culled sum opens. One
// warp per listed tile; an ascending stable sort of (key, tile) gives the order.
template <int OP>
__global__ void k_sep_tile_cost(CullArgs a, int64_t n, float reach, unsigned *key) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= n) return;   // whole warps leave together
  const CullQueries &q = a.q;
  const int t = q.tile_list[w];
  const int T = q.tile;
  const int64_t i0 = (int64_t)(t % q.ntx) * T, j0 = (int64_t)(t / q.ntx) * T;
  const int64_t i1 = (i0 + T < q.gnx ? i0 + T : q.gnx) - 1;
  const int64_t j1 = (j0 + T < q.gny ? j0 + T : q.gny) - 1;
  const float x0 = grid_coord(q.gx0, q.gdx, i0), x1 = grid_coord(q.gx0, q.gdx, i1);
  const float y0 = grid_coord(q.gy0, q.gdy, j0), y1 = grid_coord(q.gy0, q.gdy, j1);
  unsigned cnt = 0;
  if (op_gauss(OP)) {
    float e = -INFINITY;
    for (int gi = lane; gi < a.n_groups; gi += 32)
      e = fmaxf(e, a.groups[gi].lm + tile_peak<OP, 2>(a.groups[gi], x0, x1, y0, y1));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
    for (int gi = lane; gi < a.n_groups; gi += 32)
      cnt += a.groups[gi].lm + tile_peak<OP, 2>(a.groups[gi], x0, x1, y0, y1) >= e - reach;
  } else {
    for (int gi = lane; gi < a.n_groups; gi += 32)
      cnt += tile_peak<OP, 2>(a.groups[gi], x0, x1, y0, y1) > 0.f;
  }
  cnt = __reduce_add_sync(0xffffffffu, cnt);
  if (lane == 0) key[w] = ~cnt;
}

}  // namespace bbkde
