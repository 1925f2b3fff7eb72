// Culled direct sum: the pair sum over the reference tiles that can contribute,
// with a rigorous bound on the part that is skipped.
//
// References are sorted along a Morton curve (host code) and packed exactly as
// for k_pair_sum_f32x2; every run of kRefTile consecutive sorted references is a
// "reference tile" with a bounding box, its widest kernel scale and its mass.
// The queries of a block fall into QPT "slots" (slot k = the k-th query of every
// thread: a compact strip of a grid tile, or a contiguous run of Morton-sorted
// queries), each with its own bounding box. For a reference tile and a box, the
// largest value any pair can reach is, for the Gaussians, 2^e with
// e = log2(mass) + s_max * d_min^2 (d_min the distance between the boxes); for
// the Epanechnikov kernels the question is whether any pair lies inside the
// support.
//
// Every run of kGroupTiles consecutive tiles is a "tile group" with the union of
// their boxes, their widest scales and their summed mass: a group bound is at
// least the bound of each member tile, so each scan tests the groups first and
// only opens the members of groups that can matter (two-level scan; a skipped
// group counts as one skipped unit with its group bound).
//
// Gaussian blocks run three scans over the tiles:
//   1. M = the largest e over the block's box;
//   2. sum every tile with e >= M - cut (the near field);
//   3. with S_k = the smallest near-field sum in slot k, the allowance
//      A_k = max(rel * S_k, abs) and T_k = log2(A_k / n_tiles) - 1, also sum
//      every remaining tile that reaches e_k >= T_k for some slot k.
// A tile left out has 2^e_k < A_k / (2 n_tiles) for every slot, so the skipped
// part of every query q of slot k is below A_k / 2 <= max(rel * S_q, abs) / 2:
// every culled sum is within rel of the full sum, or within abs of it, whichever
// is larger (plus the FP32 arithmetic error of the full sum). abs = 0 gives the
// purely relative bound. This is the reference's combined criterion: its tree
// stops refining a query once the bounds are within rel_err relative or
// abs_err absolute (KernelDensityImpl.h:1071-1095). Tiles whose largest pair exponent s_max d_min^2 is below -128
// are skipped without a bound: ex2.approx.ftz flushes every such kernel value
// to zero, so they add exactly nothing to the FP32 sum either. The per-block
// worst ratio (skipped bound / S_k) is written for the host to verify.
// Epanechnikov blocks sum every tile that intersects the support of some slot;
// the skipped part is exactly zero.
//
// Summation is the direct kernel's: FP32 partial sums of kChunk pairs folded
// into per-query Kahan accumulators, tiles in ascending sorted order, near field
// before far field, so results are deterministic.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kde_device.cuh"

namespace bbkde {

constexpr int kRefTile = 256;      // references per culling tile
constexpr int kCullChunk = 1024;   // capacity of the per-batch list of needed tiles
constexpr int kGroupTiles = 16;    // tiles per tile group (two-level scan)

struct RefTile {
  float x0, x1, y0, y1;   // bounding box (y unused in 1-D)
  float sx, sy;           // widest (largest, i.e. least negative) scales
  float lm;               // log2 of 1.01 * sum |mass| (-inf for an empty tile)
  float pad;
};

// Where the queries of a block come from and where its results go.
//   mode 0: explicit FP32 coordinates qx/qy[0, count), block b owns queries
//           [b * QPB, (b + 1) * QPB); result i -> out[i].
//   mode 1: tiles of a regular grid: block b owns grid tile tile_list[b] of
//           tile x tile points (tiles numbered ty * ntx + tx); point (i, j) is at
//           (gx0 + i gdx, gy0 + j gdy) and its result goes to out[j * gnx + i].
struct CullQueries {
  int mode;
  const float *qx, *qy;
  int64_t count;
  const int *tile_list;
  int tile, ntx;
  int64_t gnx, gny;
  double gx0, gdx, gy0, gdy;
  double *out;
  double scale;
};

struct CullArgs {
  const float4 *refs;     // Morton-sorted packed records
  const float *extra;     // second scale column of the product kernels (or null)
  const RefTile *tiles;
  const RefTile *groups;  // one per kGroupTiles consecutive tiles (bounds of the union)
  int n_tiles;
  int n_groups;
  int64_t n_ref;
  float cut;              // near-field width in log2 units
  double rel;             // bound of the skipped part relative to the block minimum
  double abs_n;           // absolute allowance of the skipped part (unnormalised units)
  CullQueries q;
  double *blk_bound;      // per block: worst (skipped bound / slot allowance A_k)
  double *blk_smin;       // per block: smallest unnormalised sum of its queries
  int *blk_tiles;         // per block: reference tiles summed
  int *status;            // tensor-core form: set to 1 if a wait expired (or null)
};

__device__ __forceinline__ float grid_coord(double x0, double dx, int64_t i) {
  return (float)(x0 + (double)i * dx);
}

// Largest kernel value of tile t for any query in the box: log2 of it for the
// Gaussians (without the mass), the linear value for the Epanechnikov kernels.
template <int OP, int D>
__device__ __forceinline__ float tile_peak(const RefTile &t, float qx0, float qx1, float qy0,
                                           float qy1) {
  const float dx = fmaxf(0.f, fmaxf(t.x0 - qx1, qx0 - t.x1));
  const float dy = D == 2 ? fmaxf(0.f, fmaxf(t.y0 - qy1, qy0 - t.y1)) : 0.f;
  if (OP == OP_GAUSS_ISO) return t.sx * (dx * dx + dy * dy);
  if (OP == OP_GAUSS_PROD) return t.sx * dx * dx + t.sy * dy * dy;
  if (OP == OP_EPAN_ISO) return 1.f + t.sx * (dx * dx + dy * dy);
  return fminf(1.f + t.sx * dx * dx, 1.f + t.sy * dy * dy);   // both factors must be > 0
}

__host__ __device__ constexpr bool op_gauss(int op) {
  return op == OP_GAUSS_ISO || op == OP_GAUSS_PROD;
}

// Query (slot k of this thread) -> coordinates and output index; false if the
// slot is empty.
template <int D, int QPB>
__device__ __forceinline__ bool cull_query(const CullQueries &q, int64_t lq, float &x, float &y,
                                           int64_t &o) {
  if (q.mode == 0) {
    const int64_t i = (int64_t)blockIdx.x * QPB + lq;
    if (i >= q.count) return false;
    x = q.qx[i];
    y = D == 2 ? q.qy[i] : 0.f;
    o = i;
    return true;
  }
  const int t = q.tile_list[blockIdx.x];
  const int64_t tx = t % q.ntx, ty = t / q.ntx;
  const int64_t i = tx * q.tile + lq % q.tile, j = ty * q.tile + lq / q.tile;
  if (lq >= (int64_t)q.tile * q.tile || i >= q.gnx || j >= q.gny) return false;
  x = grid_coord(q.gx0, q.gdx, i);
  y = grid_coord(q.gy0, q.gdy, j);
  o = j * q.gnx + i;
  return true;
}

// Exponent below which every FP32 kernel value is flushed to zero.
constexpr float kFlushExp = -128.0f;

// Largest bound(t) over all tiles (block-wide; every thread gets the result).
// Thread-per-group: a group whose bound does not exceed the thread's running
// maximum cannot hold a tile that does, so only the others are opened.
template <int BLOCK, class Bound>
__device__ __forceinline__ float cull_max(const CullArgs &a, float *s_red, Bound bound) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float e = -INFINITY;
  for (int gi = tid; gi < a.n_groups; gi += BLOCK) {
    if (bound(a.groups[gi]) > e) {
      const int t1 = min((gi + 1) * kGroupTiles, a.n_tiles);
      for (int ti = gi * kGroupTiles; ti < t1; ++ti) e = fmaxf(e, bound(a.tiles[ti]));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
  if (lane == 0) s_red[warp] = e;
  __syncthreads();
  e = -INFINITY;
#pragma unroll
  for (int w = 0; w < BLOCK / 32; ++w) e = fmaxf(e, s_red[w]);
  __syncthreads();
  return e;
}

// Groups tested per batch of cull_pass and the length of its tile list.
__host__ __device__ constexpr int cull_groups_per_batch(int block) {
  return block < kCullChunk / kGroupTiles ? block : kCullChunk / kGroupTiles;
}
__host__ __device__ constexpr int cull_list_len(int block) {
  return cull_groups_per_batch(block) * kGroupTiles;
}

// Block-wide ordered append: the threads with pred write value to dst[rank], rank
// = the number of such threads before them; returns how many wrote (every thread).
template <int BLOCK>
__device__ __forceinline__ int block_append(bool pred, int value, int *dst, int *s_wc) {
  constexpr int NW = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, pred);
  const int rank = __popc(b & ((1u << lane) - 1u));
  if (NW == 1) {
    if (pred) dst[rank] = value;
    __syncwarp();
    return __popc(b);
  }
  if (lane == 0) s_wc[warp] = __popc(b);
  __syncthreads();
  int base = 0, total = 0;
#pragma unroll
  for (int w = 0; w < NW; ++w) {
    base += w < warp ? s_wc[w] : 0;
    total += s_wc[w];
  }
  if (pred) dst[base + rank] = value;
  __syncthreads();
  return total;
}

// One culling pass over the tiles, two levels. Each batch, thread tid < GR tests
// one group (group_needed; it also books the bound of a group it skips); the
// needed groups are listed in order (s_glist, GR entries), and the block then
// tests their members in parallel (tile_needed), BLOCK at a time. The needed
// tiles of the batch are listed in ascending order in s_list[0, total) (capacity
// cull_list_len(BLOCK)) and handed to sum_list(total), which every thread calls.
// With parts > 1 the block takes every parts-th batch from batch `part` on (the
// blocks of one tile then share its reference groups). Returns the number of
// tiles listed.
template <int BLOCK, class GroupNeeded, class TileNeeded, class SumList>
__device__ __forceinline__ int cull_pass(const CullArgs &a, int *s_list, int *s_glist, int *s_wc,
                                         GroupNeeded group_needed, TileNeeded tile_needed,
                                         SumList sum_list, int part = 0, int parts = 1) {
  constexpr int GR = cull_groups_per_batch(BLOCK);
  const int tid = threadIdx.x;
  int summed = 0;
  for (int g0 = part * GR; g0 < a.n_groups; g0 += parts * GR) {
    const int gi = g0 + tid;
    const bool gneed = tid < GR && gi < a.n_groups && group_needed(a.groups[gi]);
    const int ng = block_append<BLOCK>(gneed, gi, s_glist, s_wc);
    int total = 0;
    for (int m0 = 0; m0 < ng * kGroupTiles; m0 += BLOCK) {
      const int m = m0 + tid;
      int ti = -1;
      if (m < ng * kGroupTiles) {
        ti = s_glist[m / kGroupTiles] * kGroupTiles + m % kGroupTiles;
        if (ti >= a.n_tiles || !tile_needed(a.tiles[ti])) ti = -1;
      }
      total += block_append<BLOCK>(ti >= 0, ti, s_list + total, s_wc);
    }
    if (total > 0) sum_list(total);
    summed += total;
    __syncthreads();
  }
  return summed;
}

template <int OP, int D, int QPT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_pair_sum_culled(CullArgs a) {
  static_assert(QPT % 2 == 0 && kRefTile % BLOCK == 0 && kCullChunk % BLOCK == 0, "shape");
  constexpr int NP = QPT / 2;
  constexpr int QPB = QPT * BLOCK;
  constexpr int NW = BLOCK / 32;
  constexpr bool kExt = op_has_extra(OP) && D == 2;
  constexpr bool kGauss = op_gauss(OP);
  __shared__ float4 s_r0[kRefTile];
  __shared__ float4 s_r1[kRefTile];
  __shared__ float4 s_r2[kExt ? kRefTile : 1];
  __shared__ int s_list[cull_list_len(BLOCK)];
  __shared__ int s_glist[cull_groups_per_batch(BLOCK)];
  __shared__ int s_wc[NW];
  __shared__ float s_box[QPT][4];     // slot boxes
  __shared__ float s_th[QPT];         // slot thresholds T_k
  __shared__ float s_f[QPT][4][NW];
  __shared__ double s_d[QPT][NW];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  float2 qx[NP], qy[NP];
  float sum[QPT], comp[QPT];
  bool valid[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    float x = 0.f, y = 0.f;
    int64_t o = 0;
    valid[k] = cull_query<D, QPB>(a.q, (int64_t)k * BLOCK + tid, x, y, o);
    if (!valid[k]) { x = 0.f; y = 0.f; }
    float bx0 = valid[k] ? x : 3e38f, bx1 = valid[k] ? x : -3e38f;
    float by0 = valid[k] ? y : 3e38f, by1 = valid[k] ? y : -3e38f;
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) {
      bx0 = fminf(bx0, __shfl_xor_sync(0xffffffffu, bx0, o2));
      bx1 = fmaxf(bx1, __shfl_xor_sync(0xffffffffu, bx1, o2));
      by0 = fminf(by0, __shfl_xor_sync(0xffffffffu, by0, o2));
      by1 = fmaxf(by1, __shfl_xor_sync(0xffffffffu, by1, o2));
    }
    if (lane == 0) {
      s_f[k][0][warp] = bx0; s_f[k][1][warp] = bx1; s_f[k][2][warp] = by0; s_f[k][3][warp] = by1;
    }
    if (k & 1) { qx[k >> 1].y = x; qy[k >> 1].y = y; }
    else { qx[k >> 1].x = x; qy[k >> 1].x = y; }
    sum[k] = 0.f;
    comp[k] = 0.f;
  }
  __syncthreads();
  if (tid < QPT) {
    float v0 = 3e38f, v1 = -3e38f, v2 = 3e38f, v3 = -3e38f;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      v0 = fminf(v0, s_f[tid][0][w]); v1 = fmaxf(v1, s_f[tid][1][w]);
      v2 = fminf(v2, s_f[tid][2][w]); v3 = fmaxf(v3, s_f[tid][3][w]);
    }
    s_box[tid][0] = v0; s_box[tid][1] = v1; s_box[tid][2] = v2; s_box[tid][3] = v3;
  }
  __syncthreads();
  // Block box = union of the slot boxes.
  float qx0 = 3e38f, qx1 = -3e38f, qy0 = 3e38f, qy1 = -3e38f;
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    qx0 = fminf(qx0, s_box[k][0]); qx1 = fmaxf(qx1, s_box[k][1]);
    qy0 = fminf(qy0, s_box[k][2]); qy1 = fmaxf(qy1, s_box[k][3]);
  }

  // Scan 1 (Gaussians): largest tile bound over the block's box.
  float e_max = -INFINITY;
  if (kGauss)
    e_max = cull_max<BLOCK>(a, &s_f[0][0][0], [&](const RefTile &t) {
      return t.lm + tile_peak<OP, D>(t, qx0, qx1, qy0, qy1);
    });
  const float t_a = e_max - a.cut;

  // Skipped bound of slot k relative to its threshold: sum of 2^(e_k - T_k) < 1
  // per skipped unit (terms below 2^-126 of the threshold flush; they are
  // negligible). ex2.approx errs by ~2^-22 relative, inside the 1% mass slack.
  float skipped[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) skipped[k] = 0.f;
  int summed = 0;

  // Is tile (or group) t needed? phase 0: Epanechnikov (support of some slot);
  // phase 1: Gaussian near field; phase 2: Gaussian far field (per-slot
  // thresholds; a unit that is not needed books its per-slot bound). For a group
  // the near-field test of phase 2 is left out: a skipped group may hold tiles
  // summed in phase 1, whose bound is then booked as well (an over-estimate).
  auto needed = [&](const RefTile &t, int phase, bool group) -> bool {
    if (!kGauss) {
      bool need = false;
#pragma unroll
      for (int k = 0; k < QPT; ++k)
        need |= tile_peak<OP, D>(t, s_box[k][0], s_box[k][1], s_box[k][2], s_box[k][3]) > 0.f;
      return need;
    }
    const float pb = tile_peak<OP, D>(t, qx0, qx1, qy0, qy1);
    if (pb < kFlushExp) return false;   // every pair flushes to zero
    const bool near = t.lm + pb >= t_a;
    if (phase == 1) return near;
    if (near && !group) return false;   // already summed
    bool need = false;
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      const float pk = tile_peak<OP, D>(t, s_box[k][0], s_box[k][1], s_box[k][2], s_box[k][3]);
      need |= pk >= kFlushExp && t.lm + pk >= s_th[k];
    }
    if (!need) {
#pragma unroll
      for (int k = 0; k < QPT; ++k) {
        const float pk = tile_peak<OP, D>(t, s_box[k][0], s_box[k][1], s_box[k][2], s_box[k][3]);
        if (pk >= kFlushExp) skipped[k] += ex2_approx(t.lm + pk - s_th[k]);
      }
    }
    return need;
  };

  // Sum the listed tiles (ascending order).
  auto sum_list = [&](int running) {
    for (int li = 0; li < running; ++li) {
      const int64_t t0 = (int64_t)s_list[li] * kRefTile;
      const int64_t t1 = min(t0 + kRefTile, a.n_ref);
#pragma unroll
      for (int i = tid; i < kRefTile; i += BLOCK) {
        const int64_t rr = t0 + i;
        const float4 v = rr < t1 ? a.refs[rr] : make_float4(0.f, 0.f, 0.f, 0.f);
        if (D == 2) {
          s_r0[i] = make_float4(-v.x, -v.x, -v.y, -v.y);
          s_r1[i] = make_float4(v.z, v.z, v.w, v.w);
          if (kExt) {
            const float e = rr < t1 ? a.extra[rr] : 0.f;
            s_r2[i] = make_float4(e, e, 0.f, 0.f);
          }
        } else {
          s_r0[i] = make_float4(-v.x, -v.x, 0.f, 0.f);
          s_r1[i] = make_float4(v.y, v.y, v.z, v.z);
        }
      }
      __syncthreads();
      for (int j0 = 0; j0 < kRefTile; j0 += kChunk) {
        float2 acc[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) acc[p] = f2(0.0f);
#pragma unroll 4
        for (int j = 0; j < kChunk; ++j) {
          const float4 r0 = s_r0[j0 + j];
          const float4 r1 = s_r1[j0 + j];
          const float4 r2 = kExt ? s_r2[j0 + j] : r1;
          const float2 m = make_float2(r1.x, r1.y);
#pragma unroll
          for (int p = 0; p < NP; ++p)
            acc[p] = __ffma2_rn(m, pair_u2<OP, D>(qx[p], qy[p], r0, r1, r2), acc[p]);
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int k = 2 * p + h;
            const float v = h ? acc[p].y : acc[p].x;
            const float y = v - comp[k];
            const float t = sum[k] + y;
            comp[k] = (t - sum[k]) - y;
            sum[k] = t;
          }
        }
      }
      __syncthreads();
    }
  };

  auto pass = [&](int phase) {
    summed += cull_pass<BLOCK>(
        a, s_list, s_glist, s_wc, [&](const RefTile &g) { return needed(g, phase, true); },
        [&](const RefTile &t) { return needed(t, phase, false); }, sum_list);
  };

  double smin_all = 0.0, ratio = 0.0;
  if (kGauss) {
    pass(1);   // scan 2: near field
    // Smallest near-field sum of every slot -> slot thresholds.
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      double m = valid[k] ? (double)sum[k] - (double)comp[k] : INFINITY;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) s_d[k][warp] = m;
    }
    __syncthreads();
    if (tid < QPT) {
      double m = INFINITY;
#pragma unroll
      for (int w = 0; w < NW; ++w) m = fmin(m, s_d[tid][w]);
      // m = +inf: an empty slot needs nothing; allowance 0 (m <= 0 and no abs):
      // the slot needs every tile that does not flush to zero.
      const double allow = fmax(a.rel * m, a.abs_n);
      s_th[tid] = allow > 0.0 ? (float)(log2(allow) - log2((double)a.n_tiles)) - 1.0f
                              : -INFINITY;
      s_d[tid][0] = m;
      s_d[tid][1] = allow;
    }
    __syncthreads();
    double smk[QPT], alk[QPT];
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      smk[k] = s_d[k][0];
      alk[k] = s_d[k][1];
    }
    __syncthreads();
    pass(2);   // scan 3: far field, bound of the rest
    // Per-slot bound of the skipped part (fixed-order reduction), worst ratio to
    // the allowance: bound_k = skipped_k 2^T_k and 2^T_k = A_k / (2 n_tiles).
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      double sk = skipped[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sk += __shfl_xor_sync(0xffffffffu, sk, o);
      if (lane == 0) s_d[k][warp] = sk;
    }
    __syncthreads();
    smin_all = INFINITY;
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      double b = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) b += s_d[k][w];
      smin_all = fmin(smin_all, smk[k]);
      if (b > 0.0) ratio = fmax(ratio, b * exp2((double)s_th[k]) / alk[k]);
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
  for (int k = 0; k < QPT; ++k) {
    float x, y;
    int64_t o;
    if (cull_query<D, QPB>(a.q, (int64_t)k * BLOCK + tid, x, y, o))
      a.q.out[o] = a.q.scale * ((double)sum[k] - (double)comp[k]);
  }
}

// ---------------------------------------------------------------------------
// Building the sorted references and their tiles.
// ---------------------------------------------------------------------------

// Order-preserving map of a float to an unsigned integer (for atomic min/max).
__device__ __forceinline__ unsigned ordered_bits(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Bounding box of n points x[i * stride], y[i * stride] -> box[0..3] as ordered
// bits {min x, min y, max x, max y}; box must start as {~0, ~0, 0, 0}.
__global__ void k_bbox(const float *x, const float *y, int stride, int64_t n, unsigned *box) {
  float x0 = 3e38f, x1 = -3e38f, y0 = 3e38f, y1 = -3e38f;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float xv = x[i * stride], yv = y ? y[i * stride] : 0.f;
    x0 = fminf(x0, xv); x1 = fmaxf(x1, xv);
    y0 = fminf(y0, yv); y1 = fmaxf(y1, yv);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o));
    x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
    y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o));
    y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&box[0], ordered_bits(x0));
    atomicMin(&box[1], ordered_bits(y0));
    atomicMax(&box[2], ordered_bits(x1));
    atomicMax(&box[3], ordered_bits(y1));
  }
}

// Spread the low 16 bits of v to the even bit positions.
__device__ __forceinline__ unsigned spread16(unsigned v) {
  v &= 0xffffu;
  v = (v | (v << 8)) & 0x00ff00ffu;
  v = (v | (v << 4)) & 0x0f0f0f0fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

__device__ __forceinline__ unsigned quantize(float v, float lo, float hi, float levels) {
  const float span = hi - lo;
  const float u = span > 0.f ? (v - lo) / span : 0.f;
  return (unsigned)fminf(fmaxf(u * levels, 0.f), levels - 1.f);
}

// Morton key (2-D: 16 bits per axis interleaved; 1-D: 32-bit quantised x) and
// the identity permutation.
__global__ void k_morton(const float *x, const float *y, int stride, int64_t n,
                         const unsigned *box, unsigned *keys, int *idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float xlo = from_ordered(box[0]), ylo = from_ordered(box[1]);
  const float xhi = from_ordered(box[2]), yhi = from_ordered(box[3]);
  unsigned key;
  if (y) {
    key = spread16(quantize(x[i * stride], xlo, xhi, 65536.f)) |
          (spread16(quantize(y[i * stride], ylo, yhi, 65536.f)) << 1);
  } else {
    const float span = xhi - xlo;
    const double u = span > 0.f ? ((double)x[i * stride] - xlo) / span : 0.0;
    key = (unsigned)fmin(fmax(u * 4294967296.0, 0.0), 4294967295.0);
  }
  keys[i] = key;
  idx[i] = (int)i;
}

__global__ void k_gather_rec(const float4 *rec, const float *ext, const int *perm, int64_t n,
                             float4 *rec_out, float *ext_out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  rec_out[i] = rec[p];
  if (ext) ext_out[i] = ext[p];
}

__global__ void k_gather_xy(const float *x, const float *y, const int *perm, int64_t n,
                            float *x_out, float *y_out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  x_out[i] = x[p];
  if (y) y_out[i] = y[p];
}

__global__ void k_scatter(const double *src, const int *perm, int64_t n, double *dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[perm[i]] = src[i];
}

// One warp per tile of kRefTile sorted records.
template <int D>
__global__ void k_ref_tiles(const float4 *rec, const float *ext, int64_t n, int n_tiles,
                            RefTile *tiles) {
  const int t = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= n_tiles) return;
  float x0 = 3e38f, x1 = -3e38f, y0 = 3e38f, y1 = -3e38f, sx = -3e38f, sy = -3e38f;
  double m = 0.0;
  for (int i = lane; i < kRefTile; i += 32) {
    const int64_t r = (int64_t)t * kRefTile + i;
    if (r >= n) break;
    const float4 v = rec[r];
    const float px = v.x, py = D == 2 ? v.y : 0.f;
    const float pm = D == 2 ? v.z : v.y, ps = D == 2 ? v.w : v.z;
    x0 = fminf(x0, px); x1 = fmaxf(x1, px);
    y0 = fminf(y0, py); y1 = fmaxf(y1, py);
    sx = fmaxf(sx, ps);
    sy = fmaxf(sy, ext ? ext[r] : ps);
    m += fabs((double)pm);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o));
    x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
    y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o));
    y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    sx = fmaxf(sx, __shfl_xor_sync(0xffffffffu, sx, o));
    sy = fmaxf(sy, __shfl_xor_sync(0xffffffffu, sy, o));
    m += __shfl_xor_sync(0xffffffffu, m, o);
  }
  if (lane == 0) {
    RefTile rt;
    rt.x0 = x0; rt.x1 = x1; rt.y0 = y0; rt.y1 = y1;
    rt.sx = sx; rt.sy = sy;
    rt.lm = m > 0.0 ? (float)log2(1.01 * m) : -INFINITY;
    rt.pad = 0.f;
    tiles[t] = rt;
  }
}

// One thread per group of kGroupTiles consecutive tiles: union of the boxes,
// widest scales, log2 of the summed (already 1%-padded) masses, rounded up.
__global__ void k_ref_groups(const RefTile *tiles, int n_tiles, int n_groups,
                             RefTile *groups) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n_groups) return;
  RefTile u;
  u.x0 = 3e38f; u.x1 = -3e38f; u.y0 = 3e38f; u.y1 = -3e38f;
  u.sx = -3e38f; u.sy = -3e38f;
  double m = 0.0;
  const int t1 = min((g + 1) * kGroupTiles, n_tiles);
  for (int ti = g * kGroupTiles; ti < t1; ++ti) {
    const RefTile t = tiles[ti];
    u.x0 = fminf(u.x0, t.x0); u.x1 = fmaxf(u.x1, t.x1);
    u.y0 = fminf(u.y0, t.y0); u.y1 = fmaxf(u.y1, t.y1);
    u.sx = fmaxf(u.sx, t.sx); u.sy = fmaxf(u.sy, t.sy);
    if (t.lm > -INFINITY) m += exp2((double)t.lm);
  }
  u.lm = m > 0.0 ? nextafterf((float)log2(m), INFINITY) : -INFINITY;
  u.pad = 0.f;
  groups[g] = u;
}

// Largest skipped-bound ratio over the blocks, summed tiles.
__global__ void k_cull_stats(const double *bound, const double *smin, const int *tiles,
                             int nblk, double *out2) {
  __shared__ double s_r[256], s_t[256];
  double r = 0.0, tsum = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    r = fmax(r, bound[b]);
    tsum += (double)tiles[b];
  }
  s_r[threadIdx.x] = r;
  s_t[threadIdx.x] = tsum;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s_r[threadIdx.x] = fmax(s_r[threadIdx.x], s_r[threadIdx.x + s]);
      s_t[threadIdx.x] += s_t[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out2[0] = s_r[0];
    out2[1] = s_t[0];
  }
}

}  // namespace bbkde
