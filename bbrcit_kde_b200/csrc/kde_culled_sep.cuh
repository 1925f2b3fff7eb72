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
// Layout: block = T*T/8 threads, lane (rg, cg) = (tid / (T/4), tid % (T/4)) owns
// rows 2rg, 2rg + 1 and columns 4cg .. 4cg + 3 of the tile (8 points). Summation:
// FP32 partial sums of kChunk references (two interleaved halves) folded into
// per-point Kahan accumulators, tiles in ascending sorted order, near field
// before far field -- deterministic.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kde_culled.cuh"

namespace bbkde {

__host__ __device__ constexpr bool op_separable(int op) {
  return op == OP_GAUSS_ISO || op == OP_GAUSS_PROD || op == OP_EPAN_PROD;
}

template <int OP, int T>
__global__ void __launch_bounds__(T *T / 8, T == 32 ? 4 : 16)
    k_pair_sum_culled_sep(CullArgs a) {
  static_assert(T == 16 || T == 32, "tile edge");
  constexpr int BLOCK = T * T / 8;
  constexpr int NW = BLOCK / 32;
  constexpr int CG = T / 4;            // column groups (4 columns each)
  constexpr int RG = T / 2;            // row groups (2 rows each)
  constexpr int NS = 8;                // slots: strips of T / 8 rows
  constexpr int SUB = 64;              // references per factor sub-chunk
  constexpr int NG = BLOCK / (2 * T);  // factor teams (references split between them)
  constexpr int STG = kRefTile + 4;    // staged column stride (x and y on different banks)
  constexpr bool kGauss = op_gauss(OP);
  constexpr bool kExt = op_has_extra(OP);
  static_assert(SUB % (2 * NG) == 0 && kRefTile % SUB == 0 && (SUB / 2) % (kChunk / 2) == 0,
                "shape");
  __shared__ __align__(16) float s_c[2 * STG];     // -x | -y of the staged references
  __shared__ __align__(16) float s_s[2 * STG];     // x scale | y scale
  __shared__ __align__(16) float s_m[2 * STG];     // 1 | mass
  __shared__ __align__(16) float2 s_fx[SUB / 2 * T];   // u_x: [pair][column] (even, odd)
  __shared__ __align__(16) float2 s_fy[SUB / 2 * T];   // m u_y: [pair][row] (even, odd)
  __shared__ float s_qx[T], s_qy[T];
  __shared__ int s_list[kCullChunk];
  __shared__ int s_wc[NW];
  __shared__ float s_box[NS][4];
  __shared__ float s_th[NS];
  __shared__ unsigned s_min[NS];       // bits of the slot's smallest near-field sum (>= 0)
  __shared__ float s_red[NW];
  __shared__ double s_d[NS][NW];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int rg = tid / CG, cg = tid % CG, slot = rg / (RG / NS);
  const CullQueries &q = a.q;
  const int t = q.tile_list[blockIdx.x];
  const int64_t i0 = (int64_t)(t % q.ntx) * T, j0 = (int64_t)(t / q.ntx) * T;
  if (tid < T) {
    s_qx[tid] = grid_coord(q.gx0, q.gdx, i0 + tid);
    s_qy[tid] = grid_coord(q.gy0, q.gdy, j0 + tid);
  }
  for (int i = tid; i < kRefTile; i += BLOCK) s_m[i] = 1.0f;
  if (tid < NS) {
    // slot tid: rows j0 + tid T/8 .. + T/8 - 1 and all columns, inside the grid
    const int64_t jlo = j0 + (int64_t)tid * (T / NS);
    const int64_t jhi = (jlo + T / NS < q.gny ? jlo + T / NS : q.gny) - 1;
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
  bool valid[8];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int k = 0; k < 4; ++k)
      valid[4 * h + k] = i0 + 4 * cg + k < q.gnx && j0 + 2 * rg + h < q.gny;
  float sum[8], comp[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) { sum[k] = 0.f; comp[k] = 0.f; }

  // This thread's factor: column w or row w - T of team ft.
  const int fw = tid % (2 * T), ft = tid / (2 * T);
  const bool fx = fw < T;
  const float fq = fx ? s_qx[fw] : s_qy[fw - T];
  const int foff = fx ? 0 : STG;
  float2 *const fdst = fx ? s_fx + fw : s_fy + (fw - T);

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
    for (int sub = 0; sub < kRefTile; sub += SUB) {
#pragma unroll 4
      for (int p = ft; p < SUB / 2; p += NG) {
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
        fdst[p * T] = __fmul2_rn(m2, u);
      }
      __syncthreads();
      for (int pc = 0; pc < SUB / 2; pc += kChunk / 2) {
        float2 acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = f2(0.0f);
#pragma unroll 8
        for (int p = pc; p < pc + kChunk / 2; ++p) {
          const float4 ey = *reinterpret_cast<const float4 *>(&s_fy[p * T + 2 * rg]);
          const float4 ea = *reinterpret_cast<const float4 *>(&s_fx[p * T + 4 * cg]);
          const float4 eb = *reinterpret_cast<const float4 *>(&s_fx[p * T + 4 * cg + 2]);
          const float2 y0 = make_float2(ey.x, ey.y), y1 = make_float2(ey.z, ey.w);
          const float2 x0 = make_float2(ea.x, ea.y), x1 = make_float2(ea.z, ea.w);
          const float2 x2 = make_float2(eb.x, eb.y), x3 = make_float2(eb.z, eb.w);
          acc[0] = __ffma2_rn(y0, x0, acc[0]);
          acc[1] = __ffma2_rn(y0, x1, acc[1]);
          acc[2] = __ffma2_rn(y0, x2, acc[2]);
          acc[3] = __ffma2_rn(y0, x3, acc[3]);
          acc[4] = __ffma2_rn(y1, x0, acc[4]);
          acc[5] = __ffma2_rn(y1, x1, acc[5]);
          acc[6] = __ffma2_rn(y1, x2, acc[6]);
          acc[7] = __ffma2_rn(y1, x3, acc[7]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float v = acc[k].x + acc[k].y;
          const float y = v - comp[k];
          const float s2 = sum[k] + y;
          comp[k] = (s2 - sum[k]) - y;
          sum[k] = s2;
        }
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
        a, s_list, s_wc, [&](const RefTile &g) { return needed(g, phase, true); },
        [&](const RefTile &rt) { return needed(rt, phase, false); }, sum_list);
  };

  double smin_all = 0.0, ratio = 0.0;
  if (kGauss) {
    pass(1);   // near field
    float m = INFINITY;
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (valid[k]) m = fminf(m, fmaxf(sum[k] - comp[k], 0.f));
    if (m < INFINITY) atomicMin(&s_min[slot], __float_as_uint(m));
    __syncthreads();
    if (tid < NS) {
      const double mk = (double)__uint_as_float(s_min[tid]);
      s_th[tid] = mk > 0.0 ? (float)(log2(a.rel * mk) - log2((double)a.n_tiles)) - 1.0f
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
    smin_all = INFINITY;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double b = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) b += s_d[k][w];
      const double mk = (double)__uint_as_float(s_min[k]);
      smin_all = fmin(smin_all, mk);
      if (b > 0.0) ratio = fmax(ratio, b * exp2((double)s_th[k]) / mk);
    }
  } else {
    pass(0);
  }
  if (tid == 0) {
    a.blk_bound[blockIdx.x] = ratio;
    a.blk_smin[blockIdx.x] = smin_all;
    a.blk_tiles[blockIdx.x] = summed;
  }
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (valid[4 * h + k])
        q.out[(j0 + 2 * rg + h) * q.gnx + (i0 + 4 * cg + k)] =
            q.scale * ((double)sum[4 * h + k] - (double)comp[4 * h + k]);
}

}  // namespace bbkde
