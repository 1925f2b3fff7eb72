// Device code of the B200 direct kernel-density library.
//
// The pair sum f(q) = sum_r m_r U(q, x_r; h a_r) is the reference's eval_kernel
// (CudaDirectKde.h:126-173) re-designed for sm_100a:
//   * references are pre-packed once per (kernel, bandwidth) into float4 records
//     {x, y, m, s} (2-D) or {x, m, s, 0} (1-D) whose s folds -log2(e)/2/(h a)^2,
//     so a Gaussian pair costs 2 FADD + FMUL + FFMA + FMUL + MUFU.EX2 + FFMA;
//   * each thread owns QPT queries (register blocking) and reads every staged
//     reference record once from shared memory as a warp-wide broadcast;
//   * per-query partial sums run in FP32 over chunks of CHUNK references and are
//     folded into a Kahan-compensated FP32 pair (sum, comp); the block writes
//     (sum - comp) in FP64; reference segments are combined in FP64 in a fixed
//     order, so results do not depend on block scheduling;
//   * the FP64 variant follows the reference's CPU arithmetic (double exp).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bbkde {

// Device pair operators. kind of the packed record -> U(q, r).
enum Op : int {
  OP_GAUSS_ISO = 0,   // exp2(s * |d|^2)                       Gaussian, Gaussian conv
  OP_GAUSS_PROD = 1,  // exp2(sx dx^2 + sy dy^2)               product Gaussian, hx != hy
  OP_EPAN_ISO = 2,    // max(1 + s |d|^2, 0)                   Epanechnikov
  OP_EPAN_PROD = 3,   // max(1 + sx dx^2, 0) max(1 + sy dy^2, 0)
  OP_EPAN_CONV = 4    // prod_k c_k^3 (u_k^2 + 6 u_k + 4), u_k = |d_k| i_k, c_k = max(2-u_k,0)
};

constexpr int kChunk = 32;   // references per FP32 partial before the Kahan fold

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// (2 - u)^3 (u^2 + 6u + 4) on u = |d| / (h a) < 2, else 0. The 1/32 of the
// reference's polynomial (KernelTraits.h:338-342) is folded into the mass.
__device__ __forceinline__ float epan_conv_f(float d, float inv) {
  float u = fabsf(d) * inv;
  float c = fmaxf(2.0f - u, 0.0f);
  float q = fmaf(u, u + 6.0f, 4.0f);
  return (c * c) * (c * q);
}
__device__ __forceinline__ double epan_conv_d(double d, double inv) {
  double u = fabs(d) * inv;
  double c = fmax(2.0 - u, 0.0);
  return c * c * c * (u * u + 6.0 * u + 4.0);
}

// Unnormalised U(q, r) in FP32 for a packed record. D = 2: r = {x, y, m, s},
// e = second scale (product kernels). D = 1: r = {x, m, s, 0}.
template <int OP, int D>
__device__ __forceinline__ float pair_u(float qx, float qy, const float4 &r, float e) {
  if (D == 2) {
    float dx = qx - r.x;
    float dy = qy - r.y;
    if (OP == OP_GAUSS_ISO) {
      float d2 = fmaf(dy, dy, dx * dx);
      return ex2_approx(d2 * r.w);
    } else if (OP == OP_GAUSS_PROD) {
      float ax = dx * dx;
      float ay = dy * dy;
      return ex2_approx(fmaf(ay, e, ax * r.w));
    } else if (OP == OP_EPAN_ISO) {
      float d2 = fmaf(dy, dy, dx * dx);
      return fmaxf(fmaf(d2, r.w, 1.0f), 0.0f);
    } else if (OP == OP_EPAN_PROD) {
      float tx = fmaxf(fmaf(dx * dx, r.w, 1.0f), 0.0f);
      float ty = fmaxf(fmaf(dy * dy, e, 1.0f), 0.0f);
      return tx * ty;
    } else {  // OP_EPAN_CONV
      return epan_conv_f(dx, r.w) * epan_conv_f(dy, e);
    }
  } else {
    float dx = qx - r.x;
    if (OP == OP_GAUSS_ISO || OP == OP_GAUSS_PROD) {
      return ex2_approx((dx * dx) * r.z);
    } else if (OP == OP_EPAN_ISO || OP == OP_EPAN_PROD) {
      return fmaxf(fmaf(dx * dx, r.z, 1.0f), 0.0f);
    } else {
      return epan_conv_f(dx, r.z);
    }
  }
}

template <int D>
__device__ __forceinline__ float rec_mass(const float4 &r) { return D == 2 ? r.z : r.y; }

// FP64 record: {x, y, m, s} / {x, m, s, 0} with natural-log scales.
template <int OP, int D>
__device__ __forceinline__ double pair_u64(double qx, double qy, const double4 &r, double e) {
  if (D == 2) {
    double dx = qx - r.x;
    double dy = qy - r.y;
    if (OP == OP_GAUSS_ISO) {
      return exp((dx * dx + dy * dy) * r.w);
    } else if (OP == OP_GAUSS_PROD) {
      return exp(dx * dx * r.w + dy * dy * e);
    } else if (OP == OP_EPAN_ISO) {
      return fmax(1.0 + (dx * dx + dy * dy) * r.w, 0.0);
    } else if (OP == OP_EPAN_PROD) {
      return fmax(1.0 + dx * dx * r.w, 0.0) * fmax(1.0 + dy * dy * e, 0.0);
    } else {
      return epan_conv_d(dx, r.w) * epan_conv_d(dy, e);
    }
  } else {
    double dx = qx - r.x;
    if (OP == OP_GAUSS_ISO || OP == OP_GAUSS_PROD) {
      return exp(dx * dx * r.z);
    } else if (OP == OP_EPAN_ISO || OP == OP_EPAN_PROD) {
      return fmax(1.0 + dx * dx * r.z, 0.0);
    } else {
      return epan_conv_d(dx, r.z);
    }
  }
}

template <int D>
__device__ __forceinline__ double rec_mass64(const double4 &r) { return D == 2 ? r.z : r.y; }

__host__ __device__ constexpr bool op_has_extra(int op) {
  return op == OP_GAUSS_PROD || op == OP_EPAN_PROD || op == OP_EPAN_CONV;
}

// Arguments of one pair-sum launch. Reference records and query coordinates are
// indexed globally; the launch covers references [r_begin, r_end) split into
// gridDim.y segments of seg_len and queries [q_begin, q_begin + q_count).
struct SumArgs {
  const void *refs;        // float4* or double4*
  const void *extra;       // float* or double* (product kernels), may be null
  const void *qx;          // float* / double*
  const void *qy;          // float* / double* (unused for D = 1)
  int64_t r_begin, r_end;
  int64_t seg_len;
  int64_t q_begin, q_count;
  int exclude_self;        // self-evaluation: skip the pair r == q (same global index)
  double scale;            // multiplies each written partial
  double *out;             // [gridDim.y][q_count] partials (or final values)
  int *status;             // device error flag (0 = ok)
};

// ---------------------------------------------------------------------------
// FP32-compensated pair sum.
// grid = (ceil(q_count / (BLOCK*QPT)), segments); block = BLOCK threads.
// Thread t of block b owns queries b*BLOCK*QPT + k*BLOCK + t, k < QPT.
// ---------------------------------------------------------------------------
template <int OP, int D, int QPT, int BLOCK, int TILE>
__device__ __forceinline__ void chunk_sum(const float4 *__restrict__ s_rec,
                                          const float *__restrict__ s_ext, int j0,
                                          const float (&qx)[QPT], const float (&qy)[QPT],
                                          float (&acc)[QPT]) {
#pragma unroll 4
  for (int j = 0; j < kChunk; ++j) {
    const float4 r = s_rec[j0 + j];
    const float e = op_has_extra(OP) ? s_ext[j0 + j] : 0.0f;
    const float m = rec_mass<D>(r);
#pragma unroll
    for (int k = 0; k < QPT; ++k) acc[k] = fmaf(m, pair_u<OP, D>(qx[k], qy[k], r, e), acc[k]);
  }
}

template <int OP, int D, int QPT, int BLOCK, int TILE>
__device__ __forceinline__ void chunk_sum_diag(const float4 *__restrict__ s_rec,
                                               const float *__restrict__ s_ext, int j0,
                                               int64_t r_glob0, const int64_t (&qg)[QPT],
                                               const float (&qx)[QPT], const float (&qy)[QPT],
                                               float (&acc)[QPT]) {
  for (int j = 0; j < kChunk; ++j) {
    const float4 r = s_rec[j0 + j];
    const float e = op_has_extra(OP) ? s_ext[j0 + j] : 0.0f;
    const float m = rec_mass<D>(r);
    const int64_t rg = r_glob0 + j;
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      float u = pair_u<OP, D>(qx[k], qy[k], r, e);
      acc[k] = fmaf(rg == qg[k] ? 0.0f : m, u, acc[k]);
    }
  }
}

template <int OP, int D, int QPT, int BLOCK, int TILE, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_pair_sum_f32(SumArgs a) {
  static_assert(TILE % kChunk == 0, "tile must hold whole chunks");
  __shared__ float4 s_rec[TILE];
  __shared__ float s_ext[op_has_extra(OP) ? TILE : 1];

  const float4 *__restrict__ refs = static_cast<const float4 *>(a.refs);
  const float *__restrict__ ext = static_cast<const float *>(a.extra);
  const float *__restrict__ gqx = static_cast<const float *>(a.qx);
  const float *__restrict__ gqy = static_cast<const float *>(a.qy);

  const int tid = threadIdx.x;
  const int64_t lq0 = (int64_t)blockIdx.x * (BLOCK * QPT);
  const int64_t r_lo = a.r_begin + (int64_t)blockIdx.y * a.seg_len;
  const int64_t r_hi = min(r_lo + a.seg_len, a.r_end);

  float qx[QPT], qy[QPT], sum[QPT], comp[QPT];
  int64_t qg[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    int64_t lq = lq0 + k * BLOCK + tid;
    bool ok = lq < a.q_count;
    qg[k] = a.q_begin + lq;
    qx[k] = ok ? gqx[a.q_begin + lq] : 0.0f;
    qy[k] = (ok && D == 2) ? gqy[a.q_begin + lq] : 0.0f;
    sum[k] = 0.0f;
    comp[k] = 0.0f;
  }
  const int64_t qg_lo = a.q_begin + lq0;
  const int64_t qg_hi = qg_lo + BLOCK * QPT;

  for (int64_t t0 = r_lo; t0 < r_hi; t0 += TILE) {
    __syncthreads();
    for (int i = tid; i < TILE; i += BLOCK) {
      int64_t r = t0 + i;
      if (r < r_hi) {
        s_rec[i] = refs[r];
        if (op_has_extra(OP)) s_ext[i] = ext[r];
      } else {
        // Zero-mass padding: contributes exactly 0 for every operator.
        s_rec[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (op_has_extra(OP)) s_ext[i] = 0.0f;
      }
    }
    __syncthreads();
    const bool diag = a.exclude_self && t0 < qg_hi && qg_lo < t0 + TILE;
    for (int j0 = 0; j0 < TILE; j0 += kChunk) {
      float acc[QPT];
#pragma unroll
      for (int k = 0; k < QPT; ++k) acc[k] = 0.0f;
      if (!diag)
        chunk_sum<OP, D, QPT, BLOCK, TILE>(s_rec, s_ext, j0, qx, qy, acc);
      else
        chunk_sum_diag<OP, D, QPT, BLOCK, TILE>(s_rec, s_ext, j0, t0 + j0, qg, qx, qy, acc);
      // Kahan fold of the chunk partial.
#pragma unroll
      for (int k = 0; k < QPT; ++k) {
        float y = acc[k] - comp[k];
        float t = sum[k] + y;
        comp[k] = (t - sum[k]) - y;
        sum[k] = t;
      }
    }
  }

  double *out = a.out + (int64_t)blockIdx.y * a.q_count;
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    int64_t lq = lq0 + k * BLOCK + tid;
    if (lq < a.q_count) out[lq] = a.scale * ((double)sum[k] - (double)comp[k]);
  }
}

// ---------------------------------------------------------------------------
// FP32-compensated pair sum on packed f32x2 arithmetic (sm_100 FADD2 / FMUL2 /
// FFMA2): each instruction evaluates the same operation for two queries, so a
// Gaussian pair costs 3 packed-FP32 issue slots + 1 MUFU.EX2 instead of 6 + 1.
// The arithmetic per query is identical to k_pair_sum_f32 (same operations,
// same IEEE round-to-nearest), only issued two lanes at a time.
//
// Shared-memory records are pre-duplicated so every operand is a ready
// register pair: r0 = {-x, -x, -y, -y}, r1 = {m, m, s, s}, r2 = {e, e, _, _}
// (2-D) and r0 = {-x, -x, 0, 0}, r1 = {m, m, s, s} (1-D); q - x is evaluated as
// q + (-x), which IEEE defines identically.
// Operators: OP_GAUSS_ISO, OP_GAUSS_PROD, OP_EPAN_ISO, OP_EPAN_PROD.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

// 2^x on the FP32 pipe for two lanes, x <= 0 -- the alternative to MUFU.EX2 that
// lets the pair sum spread its exponentials over two pipes. Range reduction by the
// 1.5 * 2^23 shift (t = x + 1.5 * 2^23 holds n = round(x) in its low mantissa bits,
// f = x - n in [-1/2, 1/2] exactly), 2^f by a degree-5 polynomial (coefficients
// fitted for minimum relative error on [-1/2, 1/2] by Lawson's iteratively
// reweighted least squares: 7.5e-8 in exact arithmetic, 2.1e-7 evaluated with FP32
// FMAs), 2^n added into the exponent field (the 0x4B400000 of t shifts out of a
// 32-bit word, leaving n << 23). x is clamped at -125 so the result is a normal
// number: a pair that MUFU.EX2 flushes to zero contributes at most 2^-125 * mass.
__device__ __forceinline__ float2 exp2_poly2(float2 x) {
  x.x = fmaxf(x.x, -125.0f);
  x.y = fmaxf(x.y, -125.0f);
  const float2 t = __fadd2_rn(x, f2(12582912.0f));
  const float2 n = __fadd2_rn(t, f2(-12582912.0f));
  const float2 f = __ffma2_rn(n, f2(-1.0f), x);
  float2 p = __ffma2_rn(f2(1.327644451521337e-3f), f, f2(9.67553723603487e-3f));
  p = __ffma2_rn(p, f, f2(5.550713464617729e-2f));
  p = __ffma2_rn(p, f, f2(2.4022120237350464e-1f));
  p = __ffma2_rn(p, f, f2(6.931469440460205e-1f));
  p = __ffma2_rn(p, f, f2(1.0000001192092896f));
  return make_float2(__uint_as_float(__float_as_uint(p.x) + (__float_as_uint(t.x) << 23)),
                     __uint_as_float(__float_as_uint(p.y) + (__float_as_uint(t.y) << 23)));
}

template <int OP, int D, bool POLY = false>
__device__ __forceinline__ float2 pair_u2(const float2 qx, const float2 qy, const float4 &r0,
                                          const float4 &r1, const float4 &r2) {
  const float2 nrx = make_float2(r0.x, r0.y);
  const float2 s = make_float2(r1.z, r1.w);
  float2 dx = __fadd2_rn(qx, nrx);
  if (D == 2) {
    const float2 nry = make_float2(r0.z, r0.w);
    float2 dy = __fadd2_rn(qy, nry);
    if (OP == OP_GAUSS_ISO) {
      float2 d2 = __ffma2_rn(dy, dy, __fmul2_rn(dx, dx));
      float2 e = __fmul2_rn(d2, s);
      return POLY ? exp2_poly2(e) : make_float2(ex2_approx(e.x), ex2_approx(e.y));
    } else if (OP == OP_GAUSS_PROD) {
      const float2 sy = make_float2(r2.x, r2.y);
      float2 e = __ffma2_rn(__fmul2_rn(dy, dy), sy, __fmul2_rn(__fmul2_rn(dx, dx), s));
      return POLY ? exp2_poly2(e) : make_float2(ex2_approx(e.x), ex2_approx(e.y));
    } else if (OP == OP_EPAN_ISO) {
      float2 d2 = __ffma2_rn(dy, dy, __fmul2_rn(dx, dx));
      float2 u = __ffma2_rn(d2, s, f2(1.0f));
      return make_float2(fmaxf(u.x, 0.0f), fmaxf(u.y, 0.0f));
    } else {  // OP_EPAN_PROD
      const float2 sy = make_float2(r2.x, r2.y);
      float2 ux = __ffma2_rn(__fmul2_rn(dx, dx), s, f2(1.0f));
      float2 uy = __ffma2_rn(__fmul2_rn(dy, dy), sy, f2(1.0f));
      return __fmul2_rn(make_float2(fmaxf(ux.x, 0.0f), fmaxf(ux.y, 0.0f)),
                        make_float2(fmaxf(uy.x, 0.0f), fmaxf(uy.y, 0.0f)));
    }
  } else {
    if (OP == OP_GAUSS_ISO || OP == OP_GAUSS_PROD) {
      float2 e = __fmul2_rn(__fmul2_rn(dx, dx), s);
      return POLY ? exp2_poly2(e) : make_float2(ex2_approx(e.x), ex2_approx(e.y));
    } else {
      float2 u = __ffma2_rn(__fmul2_rn(dx, dx), s, f2(1.0f));
      return make_float2(fmaxf(u.x, 0.0f), fmaxf(u.y, 0.0f));
    }
  }
}

__host__ __device__ constexpr bool op_packed(int op) {
  return op == OP_GAUSS_ISO || op == OP_GAUSS_PROD || op == OP_EPAN_ISO || op == OP_EPAN_PROD;
}

// One reference (shared-memory record j) against this thread's query pairs.
template <int OP, int D, int NP, bool POLY, bool EXT>
__device__ __forceinline__ void ref_pairs(const float4 *s_r0, const float4 *s_r1,
                                          const float4 *s_r2, int j, const float2 (&qx)[NP],
                                          const float2 (&qy)[NP], float2 (&acc)[NP]) {
  const float4 r0 = s_r0[j];
  const float4 r1 = s_r1[j];
  const float4 r2 = EXT ? s_r2[j] : r1;
  const float2 m = make_float2(r1.x, r1.y);
#pragma unroll
  for (int p = 0; p < NP; ++p)
    acc[p] = __ffma2_rn(m, pair_u2<OP, D, POLY>(qx[p], qy[p], r0, r1, r2), acc[p]);
}

// POLY_EVERY > 0: for the Gaussians, every POLY_EVERY-th reference of a chunk takes
// its exponentials from exp2_poly2 (FP32 pipe) instead of MUFU.EX2, so that both
// pipes share the work (1 in 8 balances them: the MUFU bound alone is 16 pairs
// per clock per SM, the joint bound ~18.3).
template <int OP, int D, int QPT, int BLOCK, int TILE, int MINB, int POLY_EVERY = 0>
__global__ void __launch_bounds__(BLOCK, MINB) k_pair_sum_f32x2(SumArgs a) {
  static_assert(QPT % 2 == 0, "queries are processed in pairs");
  static_assert(kChunk % (POLY_EVERY > 0 ? POLY_EVERY : 1) == 0, "poly stride divides a chunk");
  static_assert(TILE % kChunk == 0 && TILE % BLOCK == 0, "tile shape");
  constexpr int NP = QPT / 2;
  constexpr bool kExt = op_has_extra(OP) && D == 2;
  __shared__ float4 s_r0[TILE];
  __shared__ float4 s_r1[TILE];
  __shared__ float4 s_r2[kExt ? TILE : 1];

  const float4 *__restrict__ refs = static_cast<const float4 *>(a.refs);
  const float *__restrict__ ext = static_cast<const float *>(a.extra);
  const float *__restrict__ gqx = static_cast<const float *>(a.qx);
  const float *__restrict__ gqy = static_cast<const float *>(a.qy);

  const int tid = threadIdx.x;
  const int64_t lq0 = (int64_t)blockIdx.x * (BLOCK * QPT);
  const int64_t r_lo = a.r_begin + (int64_t)blockIdx.y * a.seg_len;
  const int64_t r_hi = min(r_lo + a.seg_len, a.r_end);

  // Query pair p of this thread = local queries (2p, 2p+1) -> slots k = 2p, 2p+1.
  float2 qx[NP], qy[NP];
  float sum[QPT], comp[QPT];
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    int64_t lq = lq0 + k * BLOCK + tid;
    bool ok = lq < a.q_count;
    float x = ok ? gqx[a.q_begin + lq] : 0.0f;
    float y = (ok && D == 2) ? gqy[a.q_begin + lq] : 0.0f;
    if (k & 1) { qx[k >> 1].y = x; qy[k >> 1].y = y; }
    else { qx[k >> 1].x = x; qy[k >> 1].x = y; }
    sum[k] = 0.0f;
    comp[k] = 0.0f;
  }
  const int64_t qg_lo = a.q_begin + lq0;
  const int64_t qg_hi = qg_lo + BLOCK * QPT;

  for (int64_t t0 = r_lo; t0 < r_hi; t0 += TILE) {
    __syncthreads();
#pragma unroll
    for (int i = tid; i < TILE; i += BLOCK) {
      int64_t r = t0 + i;
      float4 v = r < r_hi ? refs[r] : make_float4(0.f, 0.f, 0.f, 0.f);  // zero-mass padding
      if (D == 2) {
        s_r0[i] = make_float4(-v.x, -v.x, -v.y, -v.y);
        s_r1[i] = make_float4(v.z, v.z, v.w, v.w);
        if (kExt) {
          float e = r < r_hi ? ext[r] : 0.0f;
          s_r2[i] = make_float4(e, e, 0.f, 0.f);
        }
      } else {
        s_r0[i] = make_float4(-v.x, -v.x, 0.f, 0.f);
        s_r1[i] = make_float4(v.y, v.y, v.z, v.z);
      }
    }
    __syncthreads();
    const bool diag = a.exclude_self && t0 < qg_hi && qg_lo < t0 + TILE;
    for (int j0 = 0; j0 < TILE; j0 += kChunk) {
      float2 acc[NP];
#pragma unroll
      for (int p = 0; p < NP; ++p) acc[p] = f2(0.0f);
      if (!diag) {
        if constexpr (POLY_EVERY == 0 || !(OP == OP_GAUSS_ISO || OP == OP_GAUSS_PROD)) {
#pragma unroll 4
          for (int j = 0; j < kChunk; ++j)
            ref_pairs<OP, D, NP, false, kExt>(s_r0, s_r1, s_r2, j0 + j, qx, qy, acc);
        } else {
#pragma unroll 1
          for (int j = 0; j < kChunk; j += POLY_EVERY) {
#pragma unroll
            for (int jj = 0; jj < POLY_EVERY - 1; ++jj)
              ref_pairs<OP, D, NP, false, kExt>(s_r0, s_r1, s_r2, j0 + j + jj, qx, qy, acc);
            ref_pairs<OP, D, NP, true, kExt>(s_r0, s_r1, s_r2, j0 + j + POLY_EVERY - 1, qx, qy,
                                             acc);
          }
        }
      } else {
        // Diagonal tile of a self-evaluation: zero the mass of the pair r == q.
        for (int j = 0; j < kChunk; ++j) {
          const float4 r0 = s_r0[j0 + j];
          const float4 r1 = s_r1[j0 + j];
          const float4 r2 = kExt ? s_r2[j0 + j] : r1;
          const int64_t rg = t0 + j0 + j;
#pragma unroll
          for (int p = 0; p < NP; ++p) {
            const int64_t q0 = qg_lo + (2 * p) * BLOCK + tid;
            const int64_t q1 = q0 + BLOCK;
            const float2 m = make_float2(rg == q0 ? 0.0f : r1.x, rg == q1 ? 0.0f : r1.y);
            acc[p] = __ffma2_rn(m, pair_u2<OP, D>(qx[p], qy[p], r0, r1, r2), acc[p]);
          }
        }
      }
#pragma unroll
      for (int p = 0; p < NP; ++p) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = 2 * p + h;
          const float v = h ? acc[p].y : acc[p].x;
          float y = v - comp[k];
          float t = sum[k] + y;
          comp[k] = (t - sum[k]) - y;
          sum[k] = t;
        }
      }
    }
  }

  double *out = a.out + (int64_t)blockIdx.y * a.q_count;
#pragma unroll
  for (int k = 0; k < QPT; ++k) {
    int64_t lq = lq0 + k * BLOCK + tid;
    if (lq < a.q_count) out[lq] = a.scale * ((double)sum[k] - (double)comp[k]);
  }
}

// ---------------------------------------------------------------------------
// FP64 pair sum (reference arithmetic). One query per thread.
// ---------------------------------------------------------------------------
template <int OP, int D, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pair_sum_f64(SumArgs a) {
  __shared__ double4 s_rec[BLOCK];
  __shared__ double s_ext[op_has_extra(OP) ? BLOCK : 1];
  const double4 *__restrict__ refs = static_cast<const double4 *>(a.refs);
  const double *__restrict__ ext = static_cast<const double *>(a.extra);
  const double *__restrict__ gqx = static_cast<const double *>(a.qx);
  const double *__restrict__ gqy = static_cast<const double *>(a.qy);

  const int tid = threadIdx.x;
  const int64_t lq = (int64_t)blockIdx.x * BLOCK + tid;
  const bool ok = lq < a.q_count;
  const int64_t qg = a.q_begin + lq;
  const double qx = ok ? gqx[qg] : 0.0;
  const double qy = (ok && D == 2) ? gqy[qg] : 0.0;
  const int64_t r_lo = a.r_begin + (int64_t)blockIdx.y * a.seg_len;
  const int64_t r_hi = min(r_lo + a.seg_len, a.r_end);

  double total = 0.0;
  for (int64_t t0 = r_lo; t0 < r_hi; t0 += BLOCK) {
    __syncthreads();
    int64_t r = t0 + tid;
    if (r < r_hi) {
      s_rec[tid] = refs[r];
      if (op_has_extra(OP)) s_ext[tid] = ext[r];
    } else {
      s_rec[tid] = make_double4(0, 0, 0, 0);
      if (op_has_extra(OP)) s_ext[tid] = 0.0;
    }
    __syncthreads();
    const int n = (int)((r_hi - t0) < BLOCK ? (r_hi - t0) : (int64_t)BLOCK);
    for (int j = 0; j < n; ++j) {
      const double4 rr = s_rec[j];
      const double e = op_has_extra(OP) ? s_ext[j] : 0.0;
      double m = rec_mass64<D>(rr);
      if (a.exclude_self && t0 + j == qg) m = 0.0;
      total += m * pair_u64<OP, D>(qx, qy, rr, e);
    }
  }
  if (ok) a.out[(int64_t)blockIdx.y * a.q_count + lq] = a.scale * total;
}

// ---------------------------------------------------------------------------
// Packing: FP64 SoA point attributes -> per-kernel records.
// ---------------------------------------------------------------------------
struct PackArgs {
  const double *x, *y, *mass, *abw;   // SoA (y unused for D = 1; abw may be null)
  int64_t n;
  int op, dim;
  double c1, c2;      // scale numerators: s = c1 / (h1 a)^2 style (see host code)
  double h1, h2;      // bandwidths
  double mass_scale;  // folded constant factor of the unnormalised kernel
};

// The record scales per operator, with a = abw_r:
//   GAUSS_*:  s = c1 / (h1 a)^2 (c1 = -log2(e)/2, or -log2(e)/4 for the
//             Gaussian convolution), e = c2 / (h2 a)^2
//   EPAN_ISO / EPAN_PROD: s = -1 / (h1 a)^2, e = -1 / (h2 a)^2
//   EPAN_CONV: s = 1 / (h1 a), e = 1 / (h2 a); mass scaled by 1/32 per dim.
__device__ __forceinline__ void pack_scales(const PackArgs &p, double a, double &s, double &e) {
  if (p.op == OP_EPAN_CONV) {
    s = 1.0 / (p.h1 * a);
    e = 1.0 / (p.h2 * a);
  } else {
    s = p.c1 / (p.h1 * p.h1 * a * a);
    e = p.c2 / (p.h2 * p.h2 * a * a);
  }
}

__global__ void k_pack_f32(PackArgs p, float4 *rec, float *ext) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  double a = p.abw ? p.abw[i] : 1.0;
  double s, e;
  pack_scales(p, a, s, e);
  float m = (float)(p.mass[i] * p.mass_scale);
  if (p.dim == 2)
    rec[i] = make_float4((float)p.x[i], (float)p.y[i], m, (float)s);
  else
    rec[i] = make_float4((float)p.x[i], m, (float)s, 0.0f);
  if (ext) ext[i] = (float)e;
}

__global__ void k_pack_f64(PackArgs p, double4 *rec, double *ext) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= p.n) return;
  double a = p.abw ? p.abw[i] : 1.0;
  double s, e;
  pack_scales(p, a, s, e);
  double m = p.mass[i] * p.mass_scale;
  if (p.dim == 2)
    rec[i] = make_double4(p.x[i], p.y[i], m, s);
  else
    rec[i] = make_double4(p.x[i], m, s, 0.0);
  if (ext) ext[i] = e;
}

__global__ void k_to_f32(const double *src, float *dst, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}

// AoS (stride dim) -> SoA columns.
__global__ void k_deinterleave(const double *aos, int dim, int64_t n, double *x, double *y) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = aos[i * dim];
  if (dim == 2) y[i] = aos[i * dim + 1];
}

__global__ void k_fill(double *dst, double v, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = v;
}

// ---------------------------------------------------------------------------
// Segment combination (+ optional weighted reductions), fixed order.
// ---------------------------------------------------------------------------
enum Epi : int { EPI_NONE = 0, EPI_W_LOG = 1, EPI_W_VALUE = 2 };

constexpr int kRedBlock = 256;

__device__ __forceinline__ double block_reduce_sum(double v, double *sm) {
  const int tid = threadIdx.x;
  sm[tid] = v;
  __syncthreads();
  for (int s = kRedBlock / 2; s > 0; s >>= 1) {
    if (tid < s) sm[tid] += sm[tid + s];
    __syncthreads();
  }
  double r = sm[0];
  __syncthreads();
  return r;
}

// out[q] = scale * sum_s partial[s][q]; with EPI_W_LOG / EPI_W_VALUE also writes
// block_sums[blockIdx.x] = sum over the block's q of w[q] * log(out[q]) / w[q] * out[q].
__global__ void __launch_bounds__(kRedBlock)
k_combine(const double *partial, int nseg, int64_t q_count, double scale, double *out,
          int epi, const double *w, double *block_sums) {
  __shared__ double sm[kRedBlock];
  int64_t q = (int64_t)blockIdx.x * kRedBlock + threadIdx.x;
  double v = 0.0;
  if (q < q_count) {
    double s = 0.0;
    for (int i = 0; i < nseg; ++i) s += partial[(int64_t)i * q_count + q];
    s *= scale;
    out[q] = s;
    if (epi == EPI_W_LOG) v = w[q] * log(s);
    else if (epi == EPI_W_VALUE) v = w[q] * s;
  }
  if (epi != EPI_NONE) {
    double b = block_reduce_sum(v, sm);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = b;
  }
}

// result[0] = sum of block_sums[0..n) in a fixed order.
__global__ void __launch_bounds__(kRedBlock)
k_sum_blocks(const double *block_sums, int64_t n, double *result) {
  __shared__ double sm[kRedBlock];
  double v = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kRedBlock) v += block_sums[i];
  double b = block_reduce_sum(v, sm);
  if (threadIdx.x == 0) result[0] = b;
}

// block_sums[b] = sum of v[i]^2 over block b's grid-stride share (fixed order).
__global__ void __launch_bounds__(kRedBlock)
k_sum_sq(const double *v, int64_t n, double *block_sums) {
  __shared__ double sm[kRedBlock];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * kRedBlock + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * kRedBlock)
    s += v[i] * v[i];
  const double b = block_reduce_sum(s, sm);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = b;
}

// Adaptive pilot finish (KernelDensityImpl.h:330-353):
// g = exp(logsum), abw_i = (pilot_i / g)^-alpha, mass_i = w_i abw_i^-dim.
__global__ void k_pilot_finalize(const double *pilot, const double *w, const double *logsum,
                                 double alpha, int dim, int64_t n, double *abw, double *mass,
                                 double *g_out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double g = exp(logsum[0]);
  if (i == 0 && g_out) g_out[0] = g;
  if (i >= n) return;
  double bw = pow(pilot[i] / g, -alpha);
  abw[i] = bw;
  mass[i] = w[i] * pow(bw, (double)-dim);
}

// sum_i w_i log(v_i) (mode 0) or sum_i w_i v_i (mode 1), v_i = f_i - sub_i C
// with sub_i rounded to FP32 (the mass the FP32 sums used; sub null: v_i = f_i),
// over n values in kWlogBlocks fixed slices: one FP64 partial per block
// (fixed-order tree within the block) -> part[blockIdx.x].
constexpr int kWlogBlocks = 256;
__global__ void k_wsum_partial(const double *f, const double *sub, double C, const double *w,
                               int mode, int64_t n, double *part) {
  __shared__ double s[256];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t lo = (int64_t)blockIdx.x * per, hi = lo + per < n ? lo + per : n;
  double acc = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = sub ? f[i] - (double)(float)sub[i] * C : f[i];
    acc += w[i] * (mode == 0 ? log(v) : v);
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// out[0] = sum of part[0, m) (m <= 1024 = blockDim.x, a power of two), fixed order.
__global__ void k_sum_partials(const double *part, int m, double *out) {
  __shared__ double s[1024];
  s[threadIdx.x] = (int)threadIdx.x < m ? part[threadIdx.x] : 0.0;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0];
}

__global__ void k_unadapt(const double *w, int64_t n, double *abw, double *mass) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  abw[i] = 1.0;
  mass[i] = w[i];
}

}  // namespace bbkde
