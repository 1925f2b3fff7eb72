// Dense query grids: surrogate predictions judged by exact sums, exact fallback.
//
// A grid of gnx x gny points (point (i, j) at (gx0 + i gdx, gy0 + j gdy), results
// row-major j * gnx + i) is cut into tile x tile blocks, numbered ty * ntx + tx.
// Per tile the pipeline decides between the surrogate's value and the exact
// (culled or full) pair sum:
//   * exact values on the half-pitch lattice: the points (a T/2, b T/2) in grid
//     index units, 0 <= a <= 2 ntx, 0 <= b <= 2 nty (the last row and column lie
//     just past the grid's end) -- one regular grid, so one factored culled sum;
//   * prediction: log-density from the network at every point; in anchored mode
//     plus the interpolation of the residual log f - net measured exactly at the
//     anchors, the even lattice points (the first point of every tile, a
//     (ntx + 1) x (nty + 1) lattice of pitch T): bilinear between the tile's
//     corners or bicubic (Catmull-Rom) over the 4 x 4 anchors around it;
//   * held-out probes, judged with the tile's own interpolant: the centre
//     (T/2, T/2), the four edge midpoints (T/2, 0), (0, T/2), (T, T/2), (T/2, T)
//     -- odd lattice points, the last two shared with the neighbouring tiles --
//     and, for 9 probes, the quarter points (T/4 + {0, T/2}, T/4 + {0, T/2}) from
//     a second lattice of pitch T/2;
//   * a tile goes exact when a probe misses by more than rel_tol, when its
//     smallest predicted density is below low_frac times the grid's largest,
//     or when a prediction or anchor is not finite.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bbkde {

struct GridDesc {
  int64_t nx, ny;
  double x0, dx, y0, dy;
  int tile, ntx, nty;
};

// Morton keys of the tile coordinates (tile order for locality of probes and
// fallback blocks).
__global__ void k_tile_keys(GridDesc g, unsigned *keys, int *ids) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ntx * g.nty) return;
  const unsigned tx = (unsigned)(t % g.ntx), ty = (unsigned)(t / g.ntx);
  unsigned k = 0;
#pragma unroll
  for (int b = 0; b < 16; ++b) k |= ((tx >> b) & 1u) << (2 * b) | ((ty >> b) & 1u) << (2 * b + 1);
  keys[t] = k;
  ids[t] = t;
}

// resid = log(exact) - net at the anchors (NaN where the exact density is not
// a positive finite number); net may be null (a zero network). Anchor (A, B),
// 0 <= A <= ntx, 0 <= B <= nty, is lattice point (2A, 2B) of the half-pitch
// lattice (row length 2 ntx + 1); resid is (ntx + 1) wide.
__global__ void k_anchor_residual(const double *exact, const float *net, int ntx, int nty,
                                  float *resid) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t aw = ntx + 1;
  if (i >= aw * (nty + 1)) return;
  const int64_t l = (2 * (i / aw)) * (2 * (int64_t)ntx + 1) + 2 * (i % aw);
  const double f = exact[l];
  const bool ok = f > 0.0 && f < INFINITY;
  resid[i] = ok ? (float)(log(f) - (net ? (double)net[l] : 0.0)) : NAN;
}

// Catmull-Rom weights of the four samples at -1, 0, 1, 2 for a point at t in [0, 1].
__device__ __forceinline__ void cr_weights(float t, float (&w)[4]) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = 0.5f * (-t3 + 2.f * t2 - t);
  w[1] = 0.5f * (3.f * t3 - 5.f * t2 + 2.f);
  w[2] = 0.5f * (-3.f * t3 + 4.f * t2 + t);
  w[3] = 0.5f * (t3 - t2);
}

// Anchor slot (a, c) of tile (tx, ty), 0 <= a, c < 4: bicubic uses the 4 x 4
// anchors around the tile (clamped at the lattice's edge), bilinear the tile's
// corners in slots 1 and 2.
__device__ __forceinline__ int64_t anchor_index(const GridDesc &g, int tx, int ty, int a, int c,
                                                int interp) {
  int ax, ay;
  if (interp == 3) {
    ax = min(max(tx - 1 + a, 0), g.ntx);
    ay = min(max(ty - 1 + c, 0), g.nty);
  } else {
    ax = tx + (a >= 2 ? 1 : 0);
    ay = ty + (c >= 2 ? 1 : 0);
  }
  return (int64_t)ay * (g.ntx + 1) + ax;
}

// Residual interpolant of one tile at tile coordinates (u, w) in [0, 1]^2
// (u = 0 at the tile's first column, u = 1 at the next tile's first column).
__device__ __forceinline__ float resid_interp(const float (&r)[4][4], float u, float w,
                                              int interp) {
  if (interp == 3) {
    float wu[4], wv[4];
    cr_weights(u, wu);
    cr_weights(w, wv);
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c)
      acc += wv[c] * (wu[0] * r[c][0] + wu[1] * r[c][1] + wu[2] * r[c][2] + wu[3] * r[c][3]);
    return acc;
  }
  return (1.f - w) * ((1.f - u) * r[1][1] + u * r[1][2]) + w * ((1.f - u) * r[2][1] + u * r[2][2]);
}

// One warp per tile (kTileReduceWarps tiles per block): pred (+)= interpolated
// residual (anchored mode; point (li, lj) of the tile at (u, w) = (li / T,
// lj / T)), tile min / max of pred, bad flag for non-finite values (a NaN anchor
// makes its tiles exact). pred_zero: pred holds zeros (it is written, not read).
constexpr int kTileReduceWarps = 8;
__global__ void __launch_bounds__(32 * kTileReduceWarps)
    k_tile_reduce(GridDesc g, float *pred, const float *resid, int interp, int pred_zero,
                  float *tmin, float *tmax, int *bad) {
  __shared__ float s_r[kTileReduceWarps][4][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int64_t t = (int64_t)blockIdx.x * kTileReduceWarps + wid;
  if (t >= (int64_t)g.ntx * g.nty) return;   // whole warps leave together
  const int tx = (int)(t % g.ntx), ty = (int)(t / g.ntx);
  if (resid && lane < 16) {
    const int a = lane & 3, c = lane >> 2;
    s_r[wid][c][a] = resid[anchor_index(g, tx, ty, a, c, interp)];
  }
  __syncwarp();
  // T (16 or 32) divides 32 * k for the lane's points l = lane + 32 k, so a lane
  // keeps one column li: the column weights fold into the four row values once.
  const int T = g.tile;
  const int tsh = T == 32 ? 5 : 4;
  const int li = lane & (T - 1);
  const float invT = 1.0f / (float)T;
  float rc[4] = {0.f, 0.f, 0.f, 0.f};   // bicubic: sum_a wu[a] r[c][a]
  float r11 = 0.f, r12 = 0.f, r21 = 0.f, r22 = 0.f;
  if (resid) {
    const float u = (float)li * invT;
    if (interp == 3) {
      float wu[4];
      cr_weights(u, wu);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        rc[c] = wu[0] * s_r[wid][c][0] + wu[1] * s_r[wid][c][1] + wu[2] * s_r[wid][c][2] +
                wu[3] * s_r[wid][c][3];
    } else {
      r11 = s_r[wid][1][1]; r12 = s_r[wid][1][2];
      r21 = s_r[wid][2][1]; r22 = s_r[wid][2][2];
    }
  }
  float mn = INFINITY, mx = -INFINITY;
  int b = 0;
  const int64_t i = (int64_t)tx * T + li;
  for (int l = lane; l < T * T; l += 32) {
    const int lj = l >> tsh;
    const int64_t j = (int64_t)ty * T + lj;
    if (i >= g.nx || j >= g.ny) continue;
    const int64_t p = j * g.nx + i;
    float v = pred_zero ? 0.f : pred[p];
    if (resid) {
      // the same interpolant as resid_interp, evaluated column-first
      const float w = (float)lj * invT;
      if (interp == 3) {
        float wv[4];
        cr_weights(w, wv);
        v += wv[0] * rc[0] + wv[1] * rc[1] + wv[2] * rc[2] + wv[3] * rc[3];
      } else {
        const float u = (float)li * invT;
        v += (1.f - w) * ((1.f - u) * r11 + u * r12) + w * ((1.f - u) * r21 + u * r22);
      }
      pred[p] = v;
    }
    if (!(v > -INFINITY && v < INFINITY)) b = 1;   // also catches NaN
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    b |= __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    tmin[t] = mn;
    tmax[t] = mx;
    bad[t] = b;
  }
}

// Smallest positive finite value of v[0, n): per block into part[blockIdx.x]
// (INFINITY if none); with final, one block over part[0, n) -> out[0] (1.0 if
// there is none). Launch: k_min_positive(v, n, part, false) on up to a few
// thousand blocks, then k_min_positive(part, blocks, out, true) on one.
__global__ void k_min_positive(const double *v, int64_t n, double *out, bool final) {
  __shared__ double s[32];
  double m = INFINITY;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double x = v[i];
    if (x > 0.0 && x < m) m = x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin(m, s[w]);
    out[blockIdx.x] = final ? (m < INFINITY ? m : 1.0) : m;
  }
}

// Largest value below +inf of v[0, n) (NaN ignored), two stages as
// k_min_positive: per block into out[blockIdx.x], then one block.
__global__ void k_max_finite(const float *v, int n, float *out) {
  __shared__ float s[32];
  float m = -INFINITY;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float x = v[i];
    if (x < INFINITY) m = fmaxf(m, x);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, s[w]);
    out[blockIdx.x] = m;
  }
}

// Probes of a tile: lattice offsets (da, db) from the tile's first lattice point
// (2 tx, 2 ty) and tile coordinates (u, w). 0: centre; 1-4: edge midpoints;
// 5-8: quarter points (on the second lattice, offsets from (2 tx, 2 ty) there).
__constant__ signed char kProbeDA[9] = {1, 1, 0, 2, 1, 0, 1, 0, 1};
__constant__ signed char kProbeDB[9] = {1, 0, 1, 1, 2, 0, 0, 1, 1};
__constant__ float kProbeU[9] = {0.5f, 0.5f, 0.f, 1.f, 0.5f, 0.25f, 0.75f, 0.25f, 0.75f};
__constant__ float kProbeW[9] = {0.5f, 0.f, 0.5f, 0.5f, 1.f, 0.25f, 0.25f, 0.75f, 0.75f};

// Inputs of the probe check: the exact values and network values (null: a zero
// network) on the half-pitch lattice ((2 ntx + 1) x (2 nty + 1)) and, for 9
// probes, on the quarter lattice (2 ntx x 2 nty); the anchor residuals (null
// outside anchored mode).
struct ProbeArgs {
  GridDesc g;
  const int *list;  // tiles to check (null: every tile)
  int64_t n_list;
  const double *lat_exact;
  const float *lat_net;
  const double *q_exact;
  const float *q_net;
  const float *resid;
  int interp;
  int probes;
  unsigned *terr;   // per tile: bits of the largest relative error (non-negative float)
};

// One thread per tile: the largest relative error of the prediction over the
// tile's probes (+inf where an exact value is not a positive finite number).
__global__ void k_probe_check(ProbeArgs a) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (a.list ? a.n_list : (int64_t)a.g.ntx * a.g.nty)) return;
  const int t = a.list ? a.list[i] : (int)i;
  const int tx = t % a.g.ntx, ty = t / a.g.ntx;
  float r[4][4];
  if (a.resid) {
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
      for (int k = 0; k < 4; ++k) r[c][k] = a.resid[anchor_index(a.g, tx, ty, k, c, a.interp)];
  }
  const int64_t lw = 2 * (int64_t)a.g.ntx + 1, qw = 2 * (int64_t)a.g.ntx;
  float err = 0.f;
  for (int k = 0; k < a.probes; ++k) {
    const bool q = k >= 5;
    const int64_t l = (2 * (int64_t)ty + kProbeDB[k]) * (q ? qw : lw) + 2 * tx + kProbeDA[k];
    const double f = q ? a.q_exact[l] : a.lat_exact[l];
    const float net = q ? (a.q_net ? a.q_net[l] : 0.f) : (a.lat_net ? a.lat_net[l] : 0.f);
    float v = net;
    if (a.resid) v += resid_interp(r, kProbeU[k], kProbeW[k], a.interp);
    float e = INFINITY;
    if (f > 0.0 && f < INFINITY) {
      e = (float)(fabs(exp((double)v) - f) / f);
      if (!(e >= 0.f)) e = INFINITY;
    }
    err = fmaxf(err, e);
  }
  a.terr[t] = __float_as_uint(err);
}

struct FlagArgs {
  GridDesc g;
  const int *order;
  const float *tmin;
  const int *bad;
  const unsigned *terr;   // may be null (no probes)
  const float *gmax;
  float log_low;          // log(low_frac)
  float rel_tol;
  int all;                // flag every tile
  int *flag;              // per tile
  int *flag_ord;          // per Morton position
  unsigned long long *counts;   // [0] low, [1] flagged, [2] max probe error bits (non-low)
};

// Counts of a warp's tiles added with one atomic per counter (lane 0).
__device__ __forceinline__ void flag_counts_add(unsigned long long *counts, bool low, bool flagged,
                                                unsigned err_bits) {
  const unsigned nl = __popc(__ballot_sync(0xffffffffu, low));
  const unsigned nf = __popc(__ballot_sync(0xffffffffu, flagged));
  const unsigned em = __reduce_max_sync(0xffffffffu, err_bits);
  if ((threadIdx.x & 31) == 0) {
    if (nl) atomicAdd(&counts[0], (unsigned long long)nl);
    if (nf) atomicAdd(&counts[1], (unsigned long long)nf);
    if (em) atomicMax(&counts[2], (unsigned long long)em);
  }
}

__global__ void k_flag_tiles(FlagArgs a) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = o < a.g.ntx * a.g.nty;   // whole warps reach the counts
  bool low = false;
  int f = 0;
  unsigned eb = 0;
  if (in) {
    const int t = a.order[o];
    f = a.all;
    if (!f) {
      low = !(a.tmin[t] >= *a.gmax + a.log_low);
      const float err = a.terr ? __uint_as_float(a.terr[t]) : 0.f;
      f = a.bad[t] || low || !(err <= a.rel_tol);
      if (!low) eb = __float_as_uint(err);
    }
    a.flag[t] = f;
    a.flag_ord[o] = f;
  }
  flag_counts_add(a.counts, low, f != 0, eb);
}

// Rescue candidates: tiles flagged by their probes alone (not low, no
// non-finite prediction), per Morton position.
__global__ void k_rescue_mark(FlagArgs a, int *cand_ord) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= a.g.ntx * a.g.nty) return;
  const int t = a.order[o];
  const bool low = !(a.tmin[t] >= *a.gmax + a.log_low);
  cand_ord[o] = a.flag[t] && !low && !a.bad[t];
}

// Coordinates of the points of the listed tiles: point l of list entry c is
// xy[c T^2 + l], (li, lj) = (l % T, l / T) (points past the grid's end included).
__global__ void k_tile_points(GridDesc g, const int *list, int64_t n, float2 *xy) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int T = g.tile;
  const int t = list[i / (T * T)];
  const int l = (int)(i % (T * T));
  const int64_t gi = (int64_t)(t % g.ntx) * T + l % T, gj = (int64_t)(t / g.ntx) * T + l / T;
  xy[i] = make_float2((float)(g.x0 + (double)gi * g.dx), (float)(g.y0 + (double)gj * g.dy));
}

// One block per listed tile: pred = network (net[c T^2 + l]) + interpolated
// residual on the tile's points; bad flag for non-finite values.
__global__ void k_tile_predict_list(GridDesc g, const int *list, const float *net,
                                    const float *resid, int interp, float *pred, int *bad) {
  __shared__ float s_r[4][4];
  __shared__ int s_bad;
  const int c = blockIdx.x, t = list[c];
  const int tx = t % g.ntx, ty = t / g.ntx;
  if (threadIdx.x < 16) {
    const int a = threadIdx.x & 3, r = threadIdx.x >> 2;
    s_r[r][a] = resid[anchor_index(g, tx, ty, a, r, interp)];
  }
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  const int T = g.tile;
  int b = 0;
  for (int l = threadIdx.x; l < T * T; l += blockDim.x) {
    const int li = l % T, lj = l / T;
    const int64_t i = (int64_t)tx * T + li, j = (int64_t)ty * T + lj;
    if (i >= g.nx || j >= g.ny) continue;
    const float v = net[(int64_t)c * T * T + l] + resid_interp(s_r, (float)li / T, (float)lj / T,
                                                                interp);
    pred[j * g.nx + i] = v;
    if (!(v > -INFINITY && v < INFINITY)) b = 1;
  }
  if (b) s_bad = 1;
  __syncthreads();
  if (threadIdx.x == 0) bad[t] = s_bad;
}

// A rescued tile keeps the network's prediction when every probe passes.
__global__ void k_rescue_update(const int *list, int64_t n, const int *bad, const unsigned *terr,
                                float rel_tol, int *flag) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int t = list[i];
  flag[t] = bad[t] || !(__uint_as_float(terr[t]) <= rel_tol);
}

// Lattice points that the rescue reads for candidate tile cand[c]: slots 0-15
// its 4 x 4 anchors (the bicubic stencil, clamped at the lattice's edge; bilinear
// reads its inner 2 x 2), slots 16-20 its centre and edge-midpoint probes. Entry
// k = c * kRescueSlots + s gets the half-pitch lattice index idx[k] and the point's
// coordinates xy[k], computed as the inference computes lattice coordinates, so
// the network values equal the whole-lattice ones.
constexpr int kRescueSlots = 21;
__global__ void k_rescue_lattice_points(GridDesc g, GridDesc gl, const int *cand, int64_t n,
                                        int64_t *idx, float2 *xy) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n * kRescueSlots) return;
  const int t = cand[k / kRescueSlots];
  const int s = (int)(k % kRescueSlots);
  const int tx = t % g.ntx, ty = t / g.ntx;
  int64_t lx, ly;
  if (s < 16) {
    lx = 2 * (int64_t)min(max(tx - 1 + (s & 3), 0), g.ntx);
    ly = 2 * (int64_t)min(max(ty - 1 + (s >> 2), 0), g.nty);
  } else {
    lx = 2 * (int64_t)tx + kProbeDA[s - 16];
    ly = 2 * (int64_t)ty + kProbeDB[s - 16];
  }
  idx[k] = ly * gl.nx + lx;
  xy[k] = make_float2((float)(gl.x0 + (double)lx * gl.dx), (float)(gl.y0 + (double)ly * gl.dy));
}

// dst[idx[k]] = v[k] (repeated indices carry equal values).
__global__ void k_scatter_net(const int64_t *idx, const float *v, int64_t n, float *dst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) dst[idx[k]] = v[k];
}

// Flags per Morton position, flagged count and largest probe error over tiles
// that are not low, from the final per-tile flags and errors (counts[1] and
// counts[2] start at 0).
__global__ void k_flag_recount(FlagArgs a) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = o < a.g.ntx * a.g.nty;   // whole warps reach the counts
  int f = 0;
  unsigned eb = 0;
  if (in) {
    const int t = a.order[o];
    f = a.flag[t];
    a.flag_ord[o] = f;
    if (a.tmin[t] >= *a.gmax + a.log_low) eb = a.terr[t];
  }
  flag_counts_add(a.counts, false, f != 0, eb);
}

// out = exp(pred) on the tiles that keep the prediction; rows over blockIdx.y,
// columns over blockIdx.x (no 64-bit division per point); tile = 1 << tshift.
__global__ void k_apply(GridDesc g, int tshift, const float *pred, const int *flag, double *out) {
  for (int64_t j = blockIdx.y; j < g.ny; j += gridDim.y) {
    const int64_t row = j * g.nx;
    const int64_t trow = (j >> tshift) * g.ntx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < g.nx;
         i += (int64_t)gridDim.x * blockDim.x) {
      if (!flag[trow + (i >> tshift)]) out[row + i] = exp((double)pred[row + i]);
    }
  }
}

}  // namespace bbkde
