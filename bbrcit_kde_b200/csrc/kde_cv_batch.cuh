// Batched cross-validation over a bandwidth grid and many datasets in one
// persistent launch (Epanechnikov product kernel).
//
// The reference evaluates one bandwidth at a time: likelihood_cross_validate
// (KernelDensityImpl.h:215-252) and lsq_convolution_cross_validate (:142-209),
// each an all-pairs self-evaluation, called in a host loop over the grid
// (grid_search/grid_search.cc:370-402). Here every (hx_a, hy_b) of the grid comes
// out of one pass over the point pairs:
//
//   Epanechnikov product: K_ab(dx, dy) = (1 - dx^2/hx_a^2)(1 - dy^2/hy_b^2) on
//   |dx| < hx_a, |dy| < hy_b. A pair with p = #{a: hx_a <= |dx|} and
//   q = #{b: hy_b <= |dy|} contributes to exactly the bandwidths a >= p, b >= q,
//   with a polynomial in (1/hx_a^2, 1/hy_b^2). So for one query i the moments
//   M_kl[p][q] = sum_j m_j dx^k dy^l (k, l in {0, 2}) binned by (p, q), then 2-D
//   inclusive prefix sums over (p, q), give
//     S_i[a][b] = P00 - P20/hx_a^2 - P02/hy_b^2 + P22/(hx_a^2 hy_b^2)
//   = sum_{j != i} m_j K_ab for all 4096 (a, b) at once; the likelihood needs
//   log(C_ab S_i[a][b]) per query, so this is done per query.
//
//   Convolution kernel (KernelTraits.h:353-357): P(u) = (2-u)^3 (u^2+6u+4)/32
//   = 1 - 5/4 u^2 + 5/8 u^3 - 1/32 u^5 on u < 2, so the same binning with the
//   16 moments {1, x^2, x^3, x^5} x {1, y^2, y^3, y^5} and cells p = #{a: 2 hx_a <= |dx|}
//   gives sum_{i,j} w_i m_j Kc_ab for all (a, b); it is linear, so it is
//   accumulated over all pairs (i < j, doubled) rather than per query.
//
// Pairs are enumerated from a uniform grid over each dataset (points sorted by
// grid cell on the host, in Morton order inside each cell), visiting only cells
// within the largest support. All arithmetic of the final scores is FP64; the
// moments are exact 64-bit fixed point.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bbkde {

constexpr int kCvMaxH = 64;                   // bandwidths per axis
constexpr int kCvCells = kCvMaxH * kCvMaxH;   // (p, q) cells
constexpr int kCvLut = 1024;                  // log2 bins of the cell lookup
constexpr int kCvMaxRanges = 2 * 8 + 1;       // candidate cell rows per query
constexpr int kCvRow = kCvMaxH + 1;           // histogram row stride (bank spread)
constexpr int kCvHist = kCvMaxH * kCvRow;     // padded (p, q) histogram size

struct CvSet {
  int64_t begin, n;          // point range in the concatenated arrays
  int64_t cell_begin;        // offset of this set's cell_start[gx * gy + 1]
  double x0, y0, inv_cell;   // grid origin and 1 / cell size
  int gx, gy;
  double diag_wm;            // sum_i w_i m_i (the i == j convolution terms)
};

// Work item: queries [q0, q1) of one set; kind 0 = likelihood / leave-one-out
// pass (part = its row in the partial buffer), kind 1..4 = convolution pass for
// x-power group kind - 1 over the queries of one grid cell (cx, cy).
struct CvItem {
  int set, kind, part, cx;
  int cy, pad;
  int64_t q0, q1;
};

struct CvArgs {
  const double *x, *y, *w, *m;      // points sorted by grid cell, concatenated
  const int64_t *cell_start;        // per set: gx * gy + 1 offsets (set-relative)
  const CvSet *sets;
  const CvItem *items;
  int n_items;
  int *counter;                     // dynamic work counter (zeroed before launch)
  int nhx, nhy;
  const double *hx, *hy;            // ascending
  const unsigned char *lutx, *luty; // lower-bound cell counts per bin of the key
  long long lut_basex, lut_basey;   // key of the first bin (see cv_cell)
  int lut_shift;                    // key = double bits >> lut_shift
  int r_epan, r_conv;               // candidate half-widths in grid cells
  double *epan_part;                // [part][2][kCvCells]: sum w log f, sum w f
  double *conv_hist;                // [set][16][kCvCells]
  unsigned long long *pairs;        // [0] likelihood pairs in support (4 atomics each),
                                    // [1] convolution pairs in support (4 per x-group)
};

// #{h[a] <= v} for v >= 0. The key (the double's bits shifted right: exponent
// and leading mantissa bits) is monotone in v; the table holds, per key bin, the
// count at the bin's lower edge, so it is a lower bound that a short exact
// correction finishes (at most one grid boundary per bin).
__device__ __forceinline__ int cv_cell(double v, const double *h, int n,
                                       const unsigned char *lut, long long base, int shift) {
  long long idx = (__double_as_longlong(v) >> shift) - base;
  idx = idx < 0 ? 0 : (idx >= kCvLut ? kCvLut - 1 : idx);
  int p = lut[idx];
  while (p < n && h[p] <= v) ++p;
  return p;
}

__device__ __forceinline__ void cv_cell_of(const CvSet &s, double x, double y, int &cx, int &cy) {
  cx = (int)floor((x - s.x0) * s.inv_cell);
  cy = (int)floor((y - s.y0) * s.inv_cell);
  cx = cx < 0 ? 0 : (cx >= s.gx ? s.gx - 1 : cx);
  cy = cy < 0 ? 0 : (cy >= s.gy ? s.gy - 1 : cy);
}

// Candidate ranges (set-relative point indices) of the grid rows within `r`
// cells of cell (cx, cy), one row per lane of warp 0, keeping only indices
// >= min_j. Empty rows stay as empty ranges. Returns through shared memory.
__device__ __forceinline__ void cv_ranges(const CvSet &s, const int64_t *cs, int cx, int cy,
                                          int r, int64_t min_j, int64_t *rb, int64_t *pre,
                                          int *nr) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const int clo = cx - r < 0 ? 0 : cx - r;
    const int chi = cx + r >= s.gx ? s.gx - 1 : cx + r;
    const int rlo = cy - r < 0 ? 0 : cy - r;
    const int rhi = cy + r >= s.gy ? s.gy - 1 : cy + r;
    const int rows = rhi - rlo + 1;   // <= 2 r + 1 <= kCvMaxRanges <= 32
    int64_t b = 0, len = 0;
    if (lane < rows) {
      const int row = rlo + lane;
      b = cs[(int64_t)row * s.gx + clo];
      int64_t e = cs[(int64_t)row * s.gx + chi + 1];
      if (b < min_j) b = min_j;
      len = e > b ? e - b : 0;
    }
    int64_t incl = len;   // inclusive warp scan of the lengths
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane < rows) {
      rb[lane] = b;
      pre[lane] = incl - len;
    }
    if (lane == rows - 1) {
      pre[rows] = incl;
      *nr = rows;
    }
  }
}

// Moments are accumulated per cell in 64-bit fixed point, normalised by the
// cell's bandwidth so every contribution lies in [0, m]: for cell p the x-part is
// x~ = |dx| / h_p (likelihood pass, |dx| < h_p) or |dx| / (2 h_p) (convolution
// pass), both < 1. Integer atomics are exact and order-independent, so results
// are bitwise reproducible; cells are converted to FP64 (times h_p^k) before the
// FP64 prefix sums.
constexpr double kCvFixLik = 4611686018427387904.0;   // 2^62: sum of masses <= 1
constexpr double kCvFixConv = 2305843009213693952.0;  // 2^61: sum of 2 w_i m_j <= 2

// Run accumulation: a thread keeps the four fixed-point moments of its latest
// cell in registers while consecutive pairs fall into the same (p, q) cell, and
// adds them to the histograms when the cell changes (and at the end of its
// pairs). Points are Morton-ordered within each grid cell, so consecutive pairs
// of a thread are spatial neighbours and share a cell wherever the bandwidth
// bins are wider than the point spacing. The sums are the same integers in
// another order: exact, and the histograms identical.
struct CvRun {
  int c = -1;
  unsigned long long a0 = 0, a1 = 0, a2 = 0, a3 = 0;
};

// Fire-and-forget shared-memory reduction (no returned value, so the warp does
// not wait for it); exact 64-bit integer addition.
__device__ __forceinline__ void cv_red(unsigned long long *h, unsigned long long iv) {
  const unsigned addr = (unsigned)__cvta_generic_to_shared(h);
  asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(addr), "l"(iv) : "memory");
}

__device__ __forceinline__ void cv_run_flush(unsigned long long *H, CvRun &r) {
  if (r.c >= 0) {
    cv_red(&H[r.c], r.a0);
    cv_red(&H[kCvHist + r.c], r.a1);
    cv_red(&H[2 * kCvHist + r.c], r.a2);
    cv_red(&H[3 * kCvHist + r.c], r.a3);
    r.c = -1;
  }
}

__device__ __forceinline__ void cv_run_add(unsigned long long *H, CvRun &r, int c, double v0,
                                           double v1, double v2, double v3) {
  const unsigned long long i0 = (unsigned long long)__double2ll_rn(v0);
  const unsigned long long i1 = (unsigned long long)__double2ll_rn(v1);
  const unsigned long long i2 = (unsigned long long)__double2ll_rn(v2);
  const unsigned long long i3 = (unsigned long long)__double2ll_rn(v3);
  if (c != r.c) {
    cv_run_flush(H, r);
    r.c = c;
    r.a0 = i0; r.a1 = i1; r.a2 = i2; r.a3 = i3;
  } else {
    r.a0 += i0; r.a1 += i1; r.a2 += i2; r.a3 += i3;
  }
}

constexpr int kCvQBlock = 256;   // queries of one convolution item (staged in smem)
constexpr int kCvUnroll = 2;     // consecutive candidates per thread and step

// Shared memory: H[4][kCvHist] (fixed point, then FP64 in place) | hx | hy |
// 1/hx | 1/hy | 1/hx^2 | 1/hy^2 | query block x, y, 2 w | ranges | misc | LUTs.
__global__ void __launch_bounds__(1024, 1) k_cv_batch(CvArgs a) {
  extern __shared__ __align__(16) double sh[];
  unsigned long long *H = reinterpret_cast<unsigned long long *>(sh);   // 4 * kCvHist
  double *Hd = sh;
  double *shx = sh + 4 * kCvHist;
  double *shy = shx + kCvMaxH;
  double *ihx = shy + kCvMaxH;
  double *ihy = ihx + kCvMaxH;
  double *ihx2 = ihy + kCvMaxH;
  double *ihy2 = ihx2 + kCvMaxH;
  double *bqx = ihy2 + kCvMaxH;        // kCvQBlock
  double *bqy = bqx + kCvQBlock;
  double *bqw = bqy + kCvQBlock;
  int64_t *rb = reinterpret_cast<int64_t *>(bqw + kCvQBlock);   // kCvMaxRanges
  int64_t *pre = rb + kCvMaxRanges;                            // kCvMaxRanges + 1
  int *misc = reinterpret_cast<int *>(pre + kCvMaxRanges + 1); // [0] item, [1] nr
  unsigned char *slutx = reinterpret_cast<unsigned char *>(misc + 4);
  unsigned char *sluty = slutx + kCvLut;

  const int tid = threadIdx.x;
  const int nt = blockDim.x;
  const int lane = tid & 31;
  for (int i = tid; i < kCvMaxH; i += nt) {
    double hx = i < a.nhx ? a.hx[i] : 1e300;
    double hy = i < a.nhy ? a.hy[i] : 1e300;
    shx[i] = hx;
    shy[i] = hy;
    ihx[i] = 1.0 / hx;
    ihy[i] = 1.0 / hy;
    ihx2[i] = 1.0 / (hx * hx);
    ihy2[i] = 1.0 / (hy * hy);
  }
  for (int i = tid; i < kCvLut; i += nt) {
    slutx[i] = a.lutx[i];
    sluty[i] = a.luty[i];
  }
  const double hxmax = a.hx[a.nhx - 1], hymax = a.hy[a.nhy - 1];
  unsigned long long n_lik = 0, n_conv = 0;   // in-support pairs of this thread
  __syncthreads();

  for (;;) {
    if (tid == 0) misc[0] = atomicAdd(a.counter, 1);
    __syncthreads();
    const int it = misc[0];
    __syncthreads();
    if (it >= a.n_items) break;
    const CvItem item = a.items[it];
    const CvSet s = a.sets[item.set];
    const int64_t *cs = a.cell_start + s.cell_begin;
    const double *X = a.x + s.begin, *Y = a.y + s.begin, *Wt = a.w + s.begin,
                 *M = a.m + s.begin;

    if (item.kind == 0) {
      // ---- likelihood / leave-one-out pass, one query at a time ----------
      // Each thread owns the cells c = tid + k * nt (k < 4) of the accumulators.
      double lik[4] = {0.0, 0.0, 0.0, 0.0}, llo[4] = {0.0, 0.0, 0.0, 0.0};
      for (int64_t i = item.q0; i < item.q1; ++i) {
        for (int c = tid; c < 4 * kCvHist; c += nt) H[c] = 0ull;
        const double qx = X[i], qy = Y[i];
        int cx, cy;
        cv_cell_of(s, qx, qy, cx, cy);
        cv_ranges(s, cs, cx, cy, a.r_epan, 0, rb, pre, misc + 1);
        __syncthreads();
        const int nr = misc[1];
        const int64_t total = pre[nr];
        int r = 0;
        CvRun run;
        for (int64_t base = (int64_t)tid * kCvUnroll; base < total;
             base += (int64_t)nt * kCvUnroll) {
          int64_t js[kCvUnroll];
          double xs[kCvUnroll], ys[kCvUnroll], ws[kCvUnroll];
#pragma unroll
          for (int u = 0; u < kCvUnroll; ++u) {
            const int64_t k = base + u;
            js[u] = -1;
            if (k < total) {
              while (k >= pre[r + 1]) ++r;
              js[u] = rb[r] + (k - pre[r]);
            }
          }
#pragma unroll
          for (int u = 0; u < kCvUnroll; ++u) {
            if (js[u] >= 0) {
              xs[u] = X[js[u]];
              ys[u] = Y[js[u]];
              ws[u] = M[js[u]];
            }
          }
#pragma unroll
          for (int u = 0; u < kCvUnroll; ++u) {
            if (js[u] < 0) continue;
            const double dx = qx - xs[u], dy = qy - ys[u];
            const double ax = fabs(dx), ay = fabs(dy);
            if (ax >= hxmax || ay >= hymax || js[u] == i) continue;
            ++n_lik;
            const int p = cv_cell(ax, shx, a.nhx, slutx, a.lut_basex, a.lut_shift);
            const int q = cv_cell(ay, shy, a.nhy, sluty, a.lut_basey, a.lut_shift);
            const int c = p * kCvRow + q;
            const double ms = ws[u] * kCvFixLik;
            const double xt = ax * ihx[p], yt = ay * ihy[q];
            const double x2 = xt * xt, y2 = yt * yt;
            cv_run_add(H, run, c, ms, ms * x2, ms * y2, ms * x2 * y2);
          }
        }
        cv_run_flush(H, run);
        __syncthreads();
        // Fixed point -> FP64 moments sum m dx^k dy^l (k, l in {0, 2}).
        for (int c = tid; c < kCvCells; c += nt) {
          const int p = c / kCvMaxH, q = c % kCvMaxH;
          const int hcell = p * kCvRow + q;
          const double hp2 = p < a.nhx ? shx[p] * shx[p] : 0.0;
          const double hq2 = q < a.nhy ? shy[q] * shy[q] : 0.0;
          const double u0 = (double)(long long)H[hcell] / kCvFixLik;
          const double u1 = (double)(long long)H[kCvHist + hcell] / kCvFixLik;
          const double u2 = (double)(long long)H[2 * kCvHist + hcell] / kCvFixLik;
          const double u3 = (double)(long long)H[3 * kCvHist + hcell] / kCvFixLik;
          Hd[hcell] = u0;
          Hd[kCvHist + hcell] = u1 * hp2;
          Hd[2 * kCvHist + hcell] = u2 * hq2;
          Hd[3 * kCvHist + hcell] = u3 * hp2 * hq2;
        }
        __syncthreads();
        // 2-D inclusive prefix: along q (rows), then along p (columns).
        for (int row = tid; row < 4 * kCvMaxH; row += nt) {
          double *hr = Hd + (row / kCvMaxH) * kCvHist + (row % kCvMaxH) * kCvRow;
          double run = 0.0;
          for (int q = 0; q < kCvMaxH; ++q) { run += hr[q]; hr[q] = run; }
        }
        __syncthreads();
        for (int col = tid; col < 4 * kCvMaxH; col += nt) {
          double *hc = Hd + (col / kCvMaxH) * kCvHist + (col % kCvMaxH);
          double run = 0.0;
          for (int p = 0; p < kCvMaxH; ++p) { run += hc[p * kCvRow]; hc[p * kCvRow] = run; }
        }
        __syncthreads();
        const double wi = Wt[i];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int c = tid + k * nt;
          if (c >= kCvCells) break;
          const int ia = c / kCvMaxH, ib = c % kCvMaxH;
          if (ia >= a.nhx || ib >= a.nhy) continue;
          const int hc = ia * kCvRow + ib;
          double S = Hd[hc] - Hd[kCvHist + hc] * ihx2[ia] - Hd[2 * kCvHist + hc] * ihy2[ib] +
                     Hd[3 * kCvHist + hc] * ihx2[ia] * ihy2[ib];
          S = S > 0.0 ? S : 0.0;
          const double f = 0.5625 / (shx[ia] * shy[ib]) * S;   // KernelTraits.h:250-252
          lik[k] += wi * log(f);
          llo[k] += wi * f;
        }
        __syncthreads();
      }
      double *dst = a.epan_part + (int64_t)item.part * 2 * kCvCells;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int c = tid + k * nt;
        if (c < kCvCells) {
          dst[c] = lik[k];
          dst[kCvCells + c] = llo[k];
        }
      }
    } else {
      // ---- convolution pass, x-power group g, one block of queries of one
      // grid cell against every candidate j > i within 2 h_max (pairs are
      // symmetric, so each unordered pair is counted once and doubled) ------
      const int g = item.kind - 1;
      const int nq = (int)(item.q1 - item.q0);
      for (int c = tid; c < 4 * kCvHist; c += nt) H[c] = 0ull;
      for (int t = tid; t < nq; t += nt) {
        bqx[t] = X[item.q0 + t];
        bqy[t] = Y[item.q0 + t];
        bqw[t] = 2.0 * Wt[item.q0 + t] * kCvFixConv;
      }
      cv_ranges(s, cs, item.cx, item.cy, a.r_conv, item.q0 + 1, rb, pre, misc + 1);
      __syncthreads();
      const int nr = misc[1];
      const int64_t total = pre[nr];
      const double hx2 = 2.0 * hxmax, hy2 = 2.0 * hymax;
      int r = 0;
      CvRun run;
      for (int64_t k = tid; k < total; k += nt) {
        while (k >= pre[r + 1]) ++r;
        const int64_t j = rb[r] + (k - pre[r]);
        const double xj = X[j], yj = Y[j], mj = M[j];
        const int64_t below = j - item.q0;                      // queries i < j
        const int lim = below < nq ? (int)below : nq;
        int t = lane % (lim > 0 ? lim : 1);                    // decorrelate lanes
        for (int s2 = 0; s2 < lim; ++s2) {
          const double ax = fabs(bqx[t] - xj), ay = fabs(bqy[t] - yj);
          const double v0 = bqw[t] * mj;
          if (++t == lim) t = 0;
          if (ax >= hx2 || ay >= hy2) continue;
          ++n_conv;
          const double hax = 0.5 * ax, hay = 0.5 * ay;
          const int p = cv_cell(hax, shx, a.nhx, slutx, a.lut_basex, a.lut_shift);
          const int q = cv_cell(hay, shy, a.nhy, sluty, a.lut_basey, a.lut_shift);
          const int c = p * kCvRow + q;
          const double xt = hax * ihx[p], yt = hay * ihy[q];   // in [0, 1)
          const double x2 = xt * xt;
          double xk = 1.0;
          if (g == 1) xk = x2;
          else if (g == 2) xk = x2 * xt;
          else if (g == 3) xk = x2 * x2 * xt;
          const double v = v0 * xk;
          const double y2 = yt * yt;
          cv_run_add(H, run, c, v, v * y2, v * y2 * yt, v * y2 * y2 * yt);
        }
      }
      cv_run_flush(H, run);
      __syncthreads();
      unsigned long long *dst = reinterpret_cast<unsigned long long *>(a.conv_hist) +
                                ((int64_t)item.set * 16 + 4 * g) * kCvCells;
      for (int e = tid; e < 4 * kCvCells; e += nt) {
        const int m4 = e / kCvCells, c = e % kCvCells;
        const unsigned long long v = H[m4 * kCvHist + (c / kCvMaxH) * kCvRow + c % kCvMaxH];
        if (v != 0ull) atomicAdd(&dst[e], v);
      }
      __syncthreads();
    }
  }
  if (a.pairs) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      n_lik += __shfl_xor_sync(0xffffffffu, n_lik, o);
      n_conv += __shfl_xor_sync(0xffffffffu, n_conv, o);
    }
    if (lane == 0) {
      atomicAdd(&a.pairs[0], n_lik);
      atomicAdd(&a.pairs[1], n_conv);
    }
  }
}

// Finalisation, one block per set: the 16 fixed-point convolution moments ->
// FP64 sum 2 w_i m_j |dx|^e_k |dy|^e_l (times (2 h_p)^e_k (2 h_q)^e_l), 2-D prefix
// in place, then per (a, b): sq = C'_ab (T_ab + sum w m), llo = sum over the
// set's likelihood items (fixed order), lsq = sq - 2 llo, lik likewise.
__global__ void __launch_bounds__(1024) k_cv_finalize(CvArgs a, const int *part_begin,
                                                      const int *part_count, double *lik_out,
                                                      double *lsq_out) {
  const int set = blockIdx.x;
  const int tid = threadIdx.x;
  const int nt = blockDim.x;
  const int ek[4] = {0, 2, 3, 5};
  double *hist = a.conv_hist + (int64_t)set * 16 * kCvCells;
  const unsigned long long *ihist = reinterpret_cast<const unsigned long long *>(hist);
  for (int e = tid; e < 16 * kCvCells; e += nt) {
    const int kx = e / (4 * kCvCells), ky = (e / kCvCells) % 4, c = e % kCvCells;
    const int p = c / kCvMaxH, q = c % kCvMaxH;
    const double sx = p < a.nhx ? pow(2.0 * a.hx[p], (double)ek[kx]) : 0.0;
    const double sy = q < a.nhy ? pow(2.0 * a.hy[q], (double)ek[ky]) : 0.0;
    hist[e] = (double)(long long)ihist[e] / kCvFixConv * sx * sy;
  }
  __syncthreads();
  for (int row = tid; row < 16 * kCvMaxH; row += nt) {
    double *hr = hist + (row / kCvMaxH) * kCvCells + (row % kCvMaxH) * kCvMaxH;
    double run = 0.0;
    for (int q = 0; q < kCvMaxH; ++q) { run += hr[q]; hr[q] = run; }
  }
  __syncthreads();
  for (int col = tid; col < 16 * kCvMaxH; col += nt) {
    double *hc = hist + (col / kCvMaxH) * kCvCells + (col % kCvMaxH);
    double run = 0.0;
    for (int p = 0; p < kCvMaxH; ++p) { run += hc[p * kCvMaxH]; hc[p * kCvMaxH] = run; }
  }
  __syncthreads();
  // P(u) = sum_k c_k u^{e_k}: (c, e) = (1, 0), (-5/4, 2), (5/8, 3), (-1/32, 5).
  const double ck[4] = {1.0, -1.25, 0.625, -0.03125};
  const double diag = a.sets[set].diag_wm;
  const int pb = part_begin[set], pc = part_count[set];
  for (int c = tid; c < kCvCells; c += nt) {
    const int ia = c / kCvMaxH, ib = c % kCvMaxH;
    if (ia >= a.nhx || ib >= a.nhy) continue;
    const double hxa = a.hx[ia], hyb = a.hy[ib];
    double T = 0.0;
    for (int kx = 0; kx < 4; ++kx) {
      const double fx = ck[kx] / pow(hxa, (double)ek[kx]);
      for (int ky = 0; ky < 4; ++ky) {
        const double fy = ck[ky] / pow(hyb, (double)ek[ky]);
        T += fx * fy * hist[(kx * 4 + ky) * kCvCells + c];
      }
    }
    const double sq = 0.36 / (hxa * hyb) * (T + diag);   // KernelTraits.h:349-351
    double lik = 0.0, llo = 0.0;
    for (int k = 0; k < pc; ++k) {
      const double *pp = a.epan_part + (int64_t)(pb + k) * 2 * kCvCells;
      lik += pp[c];
      llo += pp[kCvCells + c];
    }
    const int64_t o = ((int64_t)set * a.nhx + ia) * a.nhy + ib;
    lik_out[o] = lik;
    lsq_out[o] = sq - 2.0 * llo;
  }
}

}  // namespace bbkde
