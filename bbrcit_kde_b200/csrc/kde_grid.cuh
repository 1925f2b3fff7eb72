// Dense query grids: surrogate predictions judged by exact sums, exact fallback.
//
// A grid of gnx x gny points (point (i, j) at (gx0 + i gdx, gy0 + j gdy), results
// row-major j * gnx + i) is cut into tile x tile blocks, numbered ty * ntx + tx.
// Per tile the pipeline decides between the surrogate's value and the exact
// (culled or full) pair sum:
//   * prediction: log-density from the network at every point; in anchored mode
//     plus the bilinear interpolation of the residual log f - net measured
//     exactly at the tile corners ("anchors", a (ntx + 1) x (nty + 1) grid offset
//     by half a point spacing);
//   * held-out probes: 1, 5 or 9 grid points per tile (centre, edge midpoints,
//     quarter points), evaluated exactly and compared with the prediction;
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
// a positive finite number); net may be null (a zero network).
__global__ void k_anchor_residual(const double *exact, const float *net, int64_t n,
                                  float *resid) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double f = exact[i];
  const bool ok = f > 0.0 && f < INFINITY;
  resid[i] = ok ? (float)(log(f) - (net ? (double)net[i] : 0.0)) : NAN;
}

// Catmull-Rom weights of the four samples at -1, 0, 1, 2 for a point at t in [0, 1].
__device__ __forceinline__ void cr_weights(float t, float (&w)[4]) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = 0.5f * (-t3 + 2.f * t2 - t);
  w[1] = 0.5f * (3.f * t3 - 5.f * t2 + 2.f);
  w[2] = 0.5f * (-3.f * t3 + 4.f * t2 + t);
  w[3] = 0.5f * (t3 - t2);
}

// One block per tile: pred += interpolated residual (anchored mode: bilinear
// between the tile's 4 corner anchors, or bicubic Catmull-Rom over the 4 x 4
// anchors around the tile, clamped at the grid's edge), tile min / max of pred,
// bad flag for non-finite values (a NaN anchor makes its tiles exact).
__global__ void k_tile_reduce(GridDesc g, float *pred, const float *resid, int interp,
                              float *tmin, float *tmax, int *bad) {
  __shared__ float s_mn[32], s_mx[32];
  __shared__ int s_bad[32];
  __shared__ float s_r[4][4];
  const int t = blockIdx.x;
  const int tx = t % g.ntx, ty = t / g.ntx;
  if (resid && threadIdx.x < 16) {
    const int a = threadIdx.x & 3, c = threadIdx.x >> 2;
    int ax, ay;
    if (interp == 3) {
      ax = min(max(tx - 1 + a, 0), g.ntx);
      ay = min(max(ty - 1 + c, 0), g.nty);
    } else {   // bilinear: the corners at slots 1 and 2
      ax = tx + (a >= 2 ? 1 : 0);
      ay = ty + (c >= 2 ? 1 : 0);
    }
    s_r[c][a] = resid[(int64_t)ay * (g.ntx + 1) + ax];
  }
  __syncthreads();
  float mn = INFINITY, mx = -INFINITY;
  int b = 0;
  const int T = g.tile;
  for (int l = threadIdx.x; l < T * T; l += blockDim.x) {
    const int li = l % T, lj = l / T;
    const int64_t i = (int64_t)tx * T + li, j = (int64_t)ty * T + lj;
    if (i >= g.nx || j >= g.ny) continue;
    const int64_t p = j * g.nx + i;
    float v = pred[p];
    if (resid) {
      const float u = (li + 0.5f) / T, w = (lj + 0.5f) / T;
      if (interp == 3) {
        float wu[4], wv[4];
        cr_weights(u, wu);
        cr_weights(w, wv);
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < 4; ++c)
          acc += wv[c] * (wu[0] * s_r[c][0] + wu[1] * s_r[c][1] + wu[2] * s_r[c][2] +
                          wu[3] * s_r[c][3]);
        v += acc;
      } else {
        v += (1.f - w) * ((1.f - u) * s_r[1][1] + u * s_r[1][2]) +
             w * ((1.f - u) * s_r[2][1] + u * s_r[2][2]);
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
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) { s_mn[warp] = mn; s_mx[warp] = mx; s_bad[warp] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; ++w) {
      mn = fminf(mn, s_mn[w]);
      mx = fmaxf(mx, s_mx[w]);
      b |= s_bad[w];
    }
    tmin[t] = mn;
    tmax[t] = mx;
    bad[t] = b;
  }
}

// Largest finite value of v[0, n) -> *out (single block).
__global__ void k_max_finite(const float *v, int n, float *out) {
  __shared__ float s[32];
  float m = -INFINITY;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float x = v[i];
    if (x < INFINITY) m = fmaxf(m, x);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, s[w]);
    *out = m;
  }
}

// Probe positions in tile coordinates (u, v in [0, 1]): the centre, the edge
// midpoints, then the quarter points -- where the error of a bilinear
// interpolation between the corners peaks.
__constant__ float kProbeU[9] = {0.5f, 0.5f, 0.f, 1.f, 0.5f, 0.25f, 0.75f, 0.25f, 0.75f};
__constant__ float kProbeV[9] = {0.5f, 0.f, 0.5f, 0.5f, 1.f, 0.25f, 0.25f, 0.75f, 0.75f};

// Probe k of the tile at Morton position o -> probe index o * P + k: FP32
// coordinates and the row-major grid index of the point.
__global__ void k_make_probes(GridDesc g, const int *order, int P, float *qx, float *qy,
                              int64_t *gidx) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ntiles = (int64_t)g.ntx * g.nty;
  if (p >= ntiles * P) return;
  const int t = order[p / P];
  const int k = (int)(p % P);
  const int tx = t % g.ntx, ty = t / g.ntx;
  const int64_t i0 = (int64_t)tx * g.tile, j0 = (int64_t)ty * g.tile;
  const int64_t wr = g.nx - i0, hr = g.ny - j0;
  const int w = wr < g.tile ? (int)wr : g.tile, h = hr < g.tile ? (int)hr : g.tile;
  const int li = min(w - 1, max(0, (int)floorf(kProbeU[k] * w)));
  const int lj = min(h - 1, max(0, (int)floorf(kProbeV[k] * h)));
  const int64_t i = i0 + li, j = j0 + lj;
  qx[p] = (float)(g.x0 + (double)i * g.dx);
  qy[p] = (float)(g.y0 + (double)j * g.dy);
  gidx[p] = j * g.nx + i;
}

// Relative error of the prediction at every probe; per tile the largest, as the
// ordered bits of a non-negative float (atomicMax is exact and order-free).
__global__ void k_probe_check(const float *pred, const int64_t *gidx, const double *exact,
                              const int *order, int P, int64_t n, unsigned *terr) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double f = exact[p];
  float err = INFINITY;
  if (f > 0.0 && f < INFINITY) {
    const double v = exp((double)pred[gidx[p]]);
    err = (float)(fabs(v - f) / f);
    if (!(err >= 0.f)) err = INFINITY;
  }
  atomicMax(&terr[order[p / P]], __float_as_uint(err));
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

__global__ void k_flag_tiles(FlagArgs a) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= a.g.ntx * a.g.nty) return;
  const int t = a.order[o];
  int f = a.all;
  if (!f) {
    const bool low = !(a.tmin[t] >= *a.gmax + a.log_low);
    const float err = a.terr ? __uint_as_float(a.terr[t]) : 0.f;
    f = a.bad[t] || low || !(err <= a.rel_tol);
    if (low) atomicAdd(&a.counts[0], 1ull);
    else atomicMax(&a.counts[2], (unsigned long long)__float_as_uint(err));
  }
  if (f) atomicAdd(&a.counts[1], 1ull);
  a.flag[t] = f;
  a.flag_ord[o] = f;
}

// out = exp(pred) on the tiles that keep the prediction.
__global__ void k_apply(GridDesc g, const float *pred, const int *flag, double *out) {
  const int64_t n = g.nx * g.ny;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = p % g.nx, j = p / g.nx;
    const int t = (int)(j / g.tile) * g.ntx + (int)(i / g.tile);
    if (!flag[t]) out[p] = exp((double)pred[p]);
  }
}

}  // namespace bbkde
