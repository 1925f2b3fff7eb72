// Surrogate network for log-density: 2 -> 128 -> 128 -> 128 -> 1, SiLU.
//
// BF16 weights and activations on the tensor cores with FP32 accumulation
// (mma.sync m16n8k16) for the two 128 x 128 layers; the 2 -> 128 input layer and
// the 128 -> 1 output layer run in FP32 on the CUDA cores (K = 2 and N = 1 are
// not tensor-core shapes). A warp owns 16 points: a layer's FP32 accumulator
// fragment (16 x 128 per warp, C layout) becomes, after bias + SiLU + BF16
// packing, the next layer's A fragments directly in registers, so forward
// activations never go through memory.
//
// Parameter vector (FP32 master copy), kParams floats:
//   W1[128][2] b1[128] W2[128][128] b2[128] W3[128][128] b3[128] w4[128] b4
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace bbkde {
namespace mlp {

constexpr int kH = 128;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kH * 2;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kH * kH;
constexpr int kOffW4 = kOffB3 + kH;
constexpr int kOffB4 = kOffW4 + kH;
constexpr int kParams = kOffB4 + 1;   // 33537
// Distance between two gradient partials in floats: kParams rounded up to a
// multiple of 4, so that every partial (and its W2, W3 blocks) is 16-byte aligned.
constexpr int kPartStride = (kParams + 3) & ~3;

constexpr int kLd = kH + 8;           // padded row (bf16 elements) of smem matrices

// Input / output normalisation: x_in = (x - c) * s, y = mu + sigma * net(x_in).
struct Norm {
  float cx, cy, sx, sy;
  float mu, sigma;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t pack_raw(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// D += A (16x16, row) * B (16x8, col), BF16 inputs, FP32 accumulate.
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// z sigmoid(z) with the fast reciprocal (__fdividef, 2 ulp): for z < -88 the
// denominator is +inf and the result is -0.
__device__ __forceinline__ float silu(float z) { return __fdividef(z, 1.0f + __expf(-z)); }
// d silu / dz = s (1 + z (1 - s)), s = sigmoid(z)
__device__ __forceinline__ float silu_grad(float z) {
  float s = __fdividef(1.0f, 1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// Accumulator fragment of a 16 x 128 warp tile: acc[j][e], j = n-tile (8 columns),
// e: 0,1 -> row g, columns 8j + 2t + {0,1}; 2,3 -> row g + 8 (g = lane / 4, t = lane % 4).
struct Frag {
  float v[16][4];
};

// A fragments (k-blocks of 16) of the BF16 activations of a C-layout tile.
__device__ __forceinline__ void to_a(const Frag &f, uint32_t (&a)[8][4]) {
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
    a[kk][0] = pack_bf16(f.v[2 * kk][0], f.v[2 * kk][1]);
    a[kk][1] = pack_bf16(f.v[2 * kk][2], f.v[2 * kk][3]);
    a[kk][2] = pack_bf16(f.v[2 * kk + 1][0], f.v[2 * kk + 1][1]);
    a[kk][3] = pack_bf16(f.v[2 * kk + 1][2], f.v[2 * kk + 1][3]);
  }
}

// out = bias + A (16 x 128) * W^T, W row-major [out][in] in smem (padded rows).
__device__ __forceinline__ void layer_fwd(const uint32_t (&a)[8][4], const __nv_bfloat16 *W,
                                          const float *bias, Frag &out, int g, int t) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float b0 = bias[8 * j + 2 * t], b1 = bias[8 * j + 2 * t + 1];
    out.v[j][0] = b0;
    out.v[j][1] = b1;
    out.v[j][2] = b0;
    out.v[j][3] = b1;
  }
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const __nv_bfloat16 *row = W + (8 * j + g) * kLd + 16 * kk + 2 * t;
      const uint32_t b0 = *reinterpret_cast<const uint32_t *>(row);
      const uint32_t b1 = *reinterpret_cast<const uint32_t *>(row + 8);
      mma16816(out.v[j], a[kk], b0, b1);
    }
  }
}

// Input layer in FP32: z1 = W1 x + b1 for the two rows (points) of this lane.
__device__ __forceinline__ void layer1(const float *W1, const float *b1, float x0, float y0,
                                       float x1, float y1, Frag &z, int t) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = 8 * j + 2 * t + h;
      const float w0 = W1[2 * n], w1 = W1[2 * n + 1], bb = b1[n];
      z.v[j][h] = fmaf(w0, x0, fmaf(w1, y0, bb));
      z.v[j][2 + h] = fmaf(w0, x1, fmaf(w1, y1, bb));
    }
  }
}

__device__ __forceinline__ void silu_inplace(Frag &f) {
#pragma unroll
  for (int j = 0; j < 16; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) f.v[j][e] = silu(f.v[j][e]);
}

// Output layer: y = w4 . a3 + b4 for rows g (lo) and g + 8 (hi), reduced over the quad.
__device__ __forceinline__ void layer4(const Frag &a3, const float *w4, float b4, float &lo,
                                       float &hi, int t) {
  lo = 0.f;
  hi = 0.f;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float wa = w4[8 * j + 2 * t], wb = w4[8 * j + 2 * t + 1];
    lo = fmaf(wa, a3.v[j][0], fmaf(wb, a3.v[j][1], lo));
    hi = fmaf(wa, a3.v[j][2], fmaf(wb, a3.v[j][3], hi));
  }
  lo += __shfl_xor_sync(0xffffffffu, lo, 1);
  lo += __shfl_xor_sync(0xffffffffu, lo, 2);
  hi += __shfl_xor_sync(0xffffffffu, hi, 1);
  hi += __shfl_xor_sync(0xffffffffu, hi, 2);
  lo += b4;
  hi += b4;
}

// ---------------------------------------------------------------------------
// Inference: persistent kernel, weights staged once per block in shared memory.
// ---------------------------------------------------------------------------
struct InferArgs {
  const float *params;          // FP32 master (W1, b's, w4, b4)
  const __nv_bfloat16 *w2, *w3; // BF16 [128][128]
  Norm norm;
  const float2 *xy;             // query coordinates, or null for a grid:
  int64_t gnx;                  //   point p at (gx0 + (p % gnx) gdx, gy0 + (p / gnx) gdy)
  double gx0, gdx, gy0, gdy;
  int64_t n;
  float *out;                   // predicted log-density
};

// Two-term BF16 activations: a = hi + lo with hi = bf16(a), lo = bf16(a - hi),
// both multiplied by the same BF16 weights (relative activation error ~2^-17
// instead of 2^-9, at twice the tensor-core work).
__device__ __forceinline__ void to_a_split(const Frag &f, uint32_t (&hi)[8][4],
                                           uint32_t (&lo)[8][4]) {
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = 2 * kk + (q >> 1), e = 2 * (q & 1);
      const __nv_bfloat162 h = __floats2bfloat162_rn(f.v[j][e], f.v[j][e + 1]);
      const float2 hf = __bfloat1622float2(h);
      hi[kk][q] = *reinterpret_cast<const uint32_t *>(&h);
      lo[kk][q] = pack_bf16(f.v[j][e] - hf.x, f.v[j][e + 1] - hf.y);
    }
  }
}

__device__ __forceinline__ void layer_fwd_split(const uint32_t (&hi)[8][4],
                                                const uint32_t (&lo)[8][4],
                                                const __nv_bfloat16 *W, const float *bias,
                                                Frag &out, int g, int t) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const float b0 = bias[8 * j + 2 * t], b1 = bias[8 * j + 2 * t + 1];
    out.v[j][0] = b0;
    out.v[j][1] = b1;
    out.v[j][2] = b0;
    out.v[j][3] = b1;
  }
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const __nv_bfloat16 *row = W + (8 * j + g) * kLd + 16 * kk + 2 * t;
      const uint32_t b0 = *reinterpret_cast<const uint32_t *>(row);
      const uint32_t b1 = *reinterpret_cast<const uint32_t *>(row + 8);
      mma16816(out.v[j], lo[kk], b0, b1);
      mma16816(out.v[j], hi[kk], b0, b1);
    }
  }
}

constexpr int kInferWarps = 4;
constexpr size_t kInferSmem =
    2 * kH * kLd * sizeof(__nv_bfloat16) + (kH * 2 + 3 * kH + kH) * sizeof(float);

template <bool kSplit>
__global__ void __launch_bounds__(kInferWarps * 32) k_mlp_infer(InferArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __nv_bfloat16 *W2 = reinterpret_cast<__nv_bfloat16 *>(smem);
  __nv_bfloat16 *W3 = W2 + kH * kLd;
  float *fp = reinterpret_cast<float *>(W3 + kH * kLd);
  float *W1 = fp, *b1 = W1 + 2 * kH, *b2 = b1 + kH, *b3 = b2 + kH, *w4 = b3 + kH;
  for (int i = threadIdx.x; i < kH * kH; i += blockDim.x) {
    const int r = i / kH, c = i % kH;
    W2[r * kLd + c] = a.w2[i];
    W3[r * kLd + c] = a.w3[i];
  }
  for (int i = threadIdx.x; i < 2 * kH; i += blockDim.x) W1[i] = a.params[kOffW1 + i];
  for (int i = threadIdx.x; i < kH; i += blockDim.x) {
    b1[i] = a.params[kOffB1 + i];
    b2[i] = a.params[kOffB2 + i];
    b3[i] = a.params[kOffB3 + i];
    w4[i] = a.params[kOffW4 + i];
  }
  const float b4 = a.params[kOffB4];
  __syncthreads();
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int64_t tiles = (a.n + 15) / 16;
  const int64_t warp0 = (int64_t)blockIdx.x * kInferWarps + (threadIdx.x >> 5);
  const int64_t nwarps = (int64_t)gridDim.x * kInferWarps;
  for (int64_t tile = warp0; tile < tiles; tile += nwarps) {
    const int64_t p0 = tile * 16 + g, p1 = p0 + 8;
    float2 q0 = make_float2(0.f, 0.f), q1 = q0;
    if (a.xy) {
      if (p0 < a.n) q0 = a.xy[p0];
      if (p1 < a.n) q1 = a.xy[p1];
    } else {
      q0 = make_float2((float)(a.gx0 + (double)(p0 % a.gnx) * a.gdx),
                       (float)(a.gy0 + (double)(p0 / a.gnx) * a.gdy));
      q1 = make_float2((float)(a.gx0 + (double)(p1 % a.gnx) * a.gdx),
                       (float)(a.gy0 + (double)(p1 / a.gnx) * a.gdy));
    }
    const float x0 = (q0.x - a.norm.cx) * a.norm.sx, y0 = (q0.y - a.norm.cy) * a.norm.sy;
    const float x1 = (q1.x - a.norm.cx) * a.norm.sx, y1 = (q1.y - a.norm.cy) * a.norm.sy;
    Frag f;
    layer1(W1, b1, x0, y0, x1, y1, f, t);
    silu_inplace(f);
    if constexpr (kSplit) {
      uint32_t Ah[8][4], Al[8][4];
      to_a_split(f, Ah, Al);
      layer_fwd_split(Ah, Al, W2, b2, f, g, t);
      silu_inplace(f);
      to_a_split(f, Ah, Al);
      layer_fwd_split(Ah, Al, W3, b3, f, g, t);
    } else {
      uint32_t A[8][4];
      to_a(f, A);
      layer_fwd(A, W2, b2, f, g, t);
      silu_inplace(f);
      to_a(f, A);
      layer_fwd(A, W3, b3, f, g, t);
    }
    silu_inplace(f);
    float lo, hi;
    layer4(f, w4, b4, lo, hi, t);
    if (t == 0) {
      if (p0 < a.n) a.out[p0] = a.norm.mu + a.norm.sigma * lo;
      if (p1 < a.n) a.out[p1] = a.norm.mu + a.norm.sigma * hi;
    }
  }
}

// ---------------------------------------------------------------------------
// Training step: forward + backward of a mini-batch, per-block partial
// gradients (reduced in a fixed order by k_mlp_reduce).
// Block = 4 warps = 64 points. Loss = mean over the batch of (net - target)^2
// in normalised units.
// ---------------------------------------------------------------------------
constexpr int kTrainWarps = 4;
constexpr int kTrainPts = kTrainWarps * 16;

struct TrainArgs {
  const float *params;
  const __nv_bfloat16 *w2, *w3;
  Norm norm;
  const float2 *xy;             // training inputs
  const float *target;          // log-density targets
  const int64_t *index;         // batch -> training row
  int64_t batch;
  float *grad_part;             // [gridDim.x][kPartStride]
  float *loss_part;             // [gridDim.x]
};

// smem: W2, W3 (padded bf16) | per point (64 x kLd bf16): a1, a2, a3, z1, z2, z3 |
// xin[64][2] fp32 | small fp32 vectors.
constexpr size_t kTrainSmem =
    2 * kH * kLd * sizeof(__nv_bfloat16) + 6 * kTrainPts * kLd * sizeof(__nv_bfloat16) +
    (2 * kTrainPts + 2 * kH + 4 * kH + 64) * sizeof(float);

__device__ __forceinline__ void store_frag(__nv_bfloat16 *M, int row0, const Frag &f, int g,
                                           int t) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int c = 8 * j + 2 * t;
    *reinterpret_cast<uint32_t *>(M + (row0 + g) * kLd + c) = pack_bf16(f.v[j][0], f.v[j][1]);
    *reinterpret_cast<uint32_t *>(M + (row0 + g + 8) * kLd + c) = pack_bf16(f.v[j][2], f.v[j][3]);
  }
}

// d = dZ (16 x 128, C layout) * W (W row-major [out][in]): the gradient with
// respect to the layer's input. B fragments gather W columns.
__device__ __forceinline__ void layer_bwd_input(const Frag &dz, const __nv_bfloat16 *W, Frag &d,
                                                int g, int t) {
  uint32_t A[8][4];
  to_a(dz, A);
#pragma unroll
  for (int j = 0; j < 16; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) d.v[j][e] = 0.f;
#pragma unroll
  for (int kk = 0; kk < 8; ++kk) {
    const int k = 16 * kk + 2 * t;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int n = 8 * j + g;
      const uint32_t b0 = pack_raw(W[k * kLd + n], W[(k + 1) * kLd + n]);
      const uint32_t b1 = pack_raw(W[(k + 8) * kLd + n], W[(k + 9) * kLd + n]);
      mma16816(d.v[j], A[kk], b0, b1);
    }
  }
}

// dW[out][in] (rows [r0, r0 + 32) of this warp, columns [c0, c0 + 64)) =
// sum over the block's 64 points of dZ[p][out] * Act[p][in], both row-major
// [point][feature] in smem.
__device__ __forceinline__ void weight_grad(const __nv_bfloat16 *dZ, const __nv_bfloat16 *Act,
                                            int r0, int c0, float (&acc)[2][8][4], int g,
                                            int t) {
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.f;
#pragma unroll
  for (int kb = 0; kb < kTrainPts / 16; ++kb) {
    const int k = 16 * kb + 2 * t;
    uint32_t A[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const int m = r0 + 16 * mt + g;
      A[mt][0] = pack_raw(dZ[k * kLd + m], dZ[(k + 1) * kLd + m]);
      A[mt][1] = pack_raw(dZ[k * kLd + m + 8], dZ[(k + 1) * kLd + m + 8]);
      A[mt][2] = pack_raw(dZ[(k + 8) * kLd + m], dZ[(k + 9) * kLd + m]);
      A[mt][3] = pack_raw(dZ[(k + 8) * kLd + m + 8], dZ[(k + 9) * kLd + m + 8]);
    }
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const int n = c0 + 8 * nt + g;
      const uint32_t b0 = pack_raw(Act[k * kLd + n], Act[(k + 1) * kLd + n]);
      const uint32_t b1 = pack_raw(Act[(k + 8) * kLd + n], Act[(k + 9) * kLd + n]);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) mma16816(acc[mt][nt], A[mt], b0, b1);
    }
  }
}

__global__ void __launch_bounds__(kTrainWarps * 32) k_mlp_train(TrainArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __nv_bfloat16 *W2 = reinterpret_cast<__nv_bfloat16 *>(smem);
  __nv_bfloat16 *W3 = W2 + kH * kLd;
  __nv_bfloat16 *A1 = W3 + kH * kLd;
  __nv_bfloat16 *A2 = A1 + kTrainPts * kLd;
  __nv_bfloat16 *A3 = A2 + kTrainPts * kLd;
  __nv_bfloat16 *Z1 = A3 + kTrainPts * kLd;   // later dZ1
  __nv_bfloat16 *Z2 = Z1 + kTrainPts * kLd;   // later dZ2
  __nv_bfloat16 *Z3 = Z2 + kTrainPts * kLd;   // later dZ3
  float *xin = reinterpret_cast<float *>(Z3 + kTrainPts * kLd);   // [64][2]
  float *W1 = xin + 2 * kTrainPts;
  float *b1 = W1 + 2 * kH;
  float *b2 = b1 + kH, *b3 = b2 + kH, *w4 = b3 + kH;
  float *red = w4 + kH;   // 64 floats of block reductions
  const int tid = threadIdx.x;
  for (int i = tid; i < kH * kH; i += blockDim.x) {
    const int r = i / kH, c = i % kH;
    W2[r * kLd + c] = a.w2[i];
    W3[r * kLd + c] = a.w3[i];
  }
  for (int i = tid; i < 2 * kH; i += blockDim.x) W1[i] = a.params[kOffW1 + i];
  for (int i = tid; i < kH; i += blockDim.x) {
    b1[i] = a.params[kOffB1 + i];
    b2[i] = a.params[kOffB2 + i];
    b3[i] = a.params[kOffB3 + i];
    w4[i] = a.params[kOffW4 + i];
  }
  const float b4 = a.params[kOffB4];
  const int64_t base = (int64_t)blockIdx.x * kTrainPts;
  for (int i = tid; i < kTrainPts; i += blockDim.x) {
    float x = 0.f, y = 0.f;
    if (base + i < a.batch) {
      const float2 q = a.xy[a.index[base + i]];
      x = (q.x - a.norm.cx) * a.norm.sx;
      y = (q.y - a.norm.cy) * a.norm.sy;
    }
    xin[2 * i] = x;
    xin[2 * i + 1] = y;
  }
  __syncthreads();

  const int warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int row0 = warp * 16;   // this warp's points within the block
  const int64_t p0 = base + row0 + g, p1 = p0 + 8;
  const bool v0 = p0 < a.batch, v1 = p1 < a.batch;
  const float inv_b = 1.0f / (float)a.batch;

  // ---- forward ----
  Frag f, z;
  uint32_t A[8][4];
  layer1(W1, b1, xin[2 * (row0 + g)], xin[2 * (row0 + g) + 1], xin[2 * (row0 + g + 8)],
         xin[2 * (row0 + g + 8) + 1], z, t);
  store_frag(Z1, row0, z, g, t);
  f = z;
  silu_inplace(f);
  store_frag(A1, row0, f, g, t);
  to_a(f, A);
  layer_fwd(A, W2, b2, z, g, t);
  store_frag(Z2, row0, z, g, t);
  f = z;
  silu_inplace(f);
  store_frag(A2, row0, f, g, t);
  to_a(f, A);
  layer_fwd(A, W3, b3, z, g, t);
  store_frag(Z3, row0, z, g, t);
  f = z;
  silu_inplace(f);
  store_frag(A3, row0, f, g, t);
  float ylo, yhi;
  layer4(f, w4, b4, ylo, yhi, t);

  // ---- loss and output-layer gradient (normalised units) ----
  float tlo = 0.f, thi = 0.f;
  if (v0) tlo = (a.target[a.index[p0]] - a.norm.mu) / a.norm.sigma;
  if (v1) thi = (a.target[a.index[p1]] - a.norm.mu) / a.norm.sigma;
  const float elo = v0 ? ylo - tlo : 0.f, ehi = v1 ? yhi - thi : 0.f;
  const float dlo = 2.f * elo * inv_b, dhi = 2.f * ehi * inv_b;   // dL/dy

  // dz3 = dy * w4 * silu'(z3); keep in registers (C layout) and in Z3 (bf16).
  Frag dz;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = 8 * j + 2 * t + h;
      dz.v[j][h] = dlo * w4[n] * silu_grad(z.v[j][h]);
      dz.v[j][2 + h] = dhi * w4[n] * silu_grad(z.v[j][2 + h]);
    }
  }
  __syncwarp();
  store_frag(Z3, row0, dz, g, t);
  // dz2 = (dz3 W3) * silu'(z2)
  Frag d;
  layer_bwd_input(dz, W3, d, g, t);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int c = 8 * j + 2 * t;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      d.v[j][h] *= silu_grad(__bfloat162float(Z2[(row0 + g) * kLd + c + h]));
      d.v[j][2 + h] *= silu_grad(__bfloat162float(Z2[(row0 + g + 8) * kLd + c + h]));
    }
  }
  __syncwarp();
  store_frag(Z2, row0, d, g, t);
  // dz1 = (dz2 W2) * silu'(z1)
  Frag d1;
  layer_bwd_input(d, W2, d1, g, t);
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int c = 8 * j + 2 * t;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      d1.v[j][h] *= silu_grad(__bfloat162float(Z1[(row0 + g) * kLd + c + h]));
      d1.v[j][2 + h] *= silu_grad(__bfloat162float(Z1[(row0 + g + 8) * kLd + c + h]));
    }
  }
  __syncwarp();
  store_frag(Z1, row0, d1, g, t);
  __syncthreads();

  // ---- weight gradients: dW3 = dZ3^T A2, dW2 = dZ2^T A1 on the tensor cores ----
  float *gp = a.grad_part + (int64_t)blockIdx.x * kPartStride;
  const int r0 = warp * 32;
  for (int layer = 0; layer < 2; ++layer) {
    const __nv_bfloat16 *dZ = layer == 0 ? Z3 : Z2;
    const __nv_bfloat16 *Act = layer == 0 ? A2 : A1;
    float *dst = gp + (layer == 0 ? kOffW3 : kOffW2);
    for (int half = 0; half < 2; ++half) {
      float acc[2][8][4];
      weight_grad(dZ, Act, r0, 64 * half, acc, g, t);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          const int m = r0 + 16 * mt + g, n = 64 * half + 8 * nt + 2 * t;
          dst[m * kH + n] = acc[mt][nt][0];
          dst[m * kH + n + 1] = acc[mt][nt][1];
          dst[(m + 8) * kH + n] = acc[mt][nt][2];
          dst[(m + 8) * kH + n + 1] = acc[mt][nt][3];
        }
    }
  }
  // ---- vectors on the CUDA cores: db1..3, dW1, dw4, db4 (fixed-order sums) ----
  for (int n = tid; n < kH; n += blockDim.x) {
    float s1 = 0.f, s2 = 0.f, s3 = 0.f, w1x = 0.f, w1y = 0.f;
    for (int p = 0; p < kTrainPts; ++p) {
      const float g1 = __bfloat162float(Z1[p * kLd + n]);
      s1 += g1;
      s2 += __bfloat162float(Z2[p * kLd + n]);
      s3 += __bfloat162float(Z3[p * kLd + n]);
      w1x += g1 * xin[2 * p];
      w1y += g1 * xin[2 * p + 1];
    }
    gp[kOffB1 + n] = s1;
    gp[kOffB2 + n] = s2;
    gp[kOffB3 + n] = s3;
    gp[kOffW1 + 2 * n] = w1x;
    gp[kOffW1 + 2 * n + 1] = w1y;
  }
  // dw4[n] = sum_p dy_p * a3[p][n]; db4 = sum_p dy_p; loss = sum_p e_p^2 / batch.
  if (t == 0) {
    red[row0 + g] = dlo;
    red[row0 + g + 8] = dhi;
  }
  __syncthreads();
  for (int n = tid; n < kH; n += blockDim.x) {
    float s = 0.f;
    for (int p = 0; p < kTrainPts; ++p) s += red[p] * __bfloat162float(A3[p * kLd + n]);
    gp[kOffW4 + n] = s;
  }
  __syncthreads();
  if (t == 0) {
    red[row0 + g] = elo * elo;
    red[row0 + g + 8] = ehi * ehi;
  }
  __syncthreads();
  if (tid == 0) {
    float s = 0.f;
    for (int p = 0; p < kTrainPts; ++p) s += red[p];
    a.loss_part[blockIdx.x] = s * inv_b;
  }
  __syncthreads();
  if (t == 0) {
    red[row0 + g] = dlo;
    red[row0 + g + 8] = dhi;
  }
  __syncthreads();
  if (tid == 0) {
    float s = 0.f;
    for (int p = 0; p < kTrainPts; ++p) s += red[p];
    gp[kOffB4] = s;
  }
}

// Sum the block partials in a fixed order; optionally apply an Adam step.
struct AdamArgs {
  const float *grad_part;
  int nparts;
  const float *loss_part;
  float *params;                // FP32 master (updated when step > 0)
  float *m, *v;                 // Adam moments
  __nv_bfloat16 *w2, *w3;       // BF16 copies refreshed from the master
  float *grad_out;              // summed gradient (may be null)
  float *loss_out;              // summed loss (may be null)
  float lr, beta1, beta2, eps;
  int step;                     // 1-based Adam step; 0 = reduce only
};

__global__ void k_mlp_reduce(AdamArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0 && a.loss_out) {
    float s = 0.f;
    for (int k = 0; k < a.nparts; ++k) s += a.loss_part[k];
    *a.loss_out = s;
  }
  if (i >= kParams) return;
  float gsum = 0.f;
  for (int k = 0; k < a.nparts; ++k) gsum += a.grad_part[(int64_t)k * kPartStride + i];
  if (a.grad_out) a.grad_out[i] = gsum;
  if (a.step > 0) {
    float m = a.beta1 * a.m[i] + (1.f - a.beta1) * gsum;
    float v = a.beta2 * a.v[i] + (1.f - a.beta2) * gsum * gsum;
    a.m[i] = m;
    a.v[i] = v;
    const float mh = m / (1.f - powf(a.beta1, (float)a.step));
    const float vh = v / (1.f - powf(a.beta2, (float)a.step));
    a.params[i] -= a.lr * mh / (sqrtf(vh) + a.eps);
  }
  const float p = a.params[i];
  if (i >= kOffW2 && i < kOffW2 + kH * kH) a.w2[i - kOffW2] = __float2bfloat16_rn(p);
  if (i >= kOffW3 && i < kOffW3 + kH * kH) a.w3[i - kOffW3] = __float2bfloat16_rn(p);
}

// Batch indices for step `step`: splitmix64 of (seed, step, i) modulo n.
__global__ void k_mlp_batch(int64_t *index, int64_t batch, int64_t n, uint64_t seed,
                            uint64_t step) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= batch) return;
  uint64_t z = seed + (step * 0x100000001B3ull + (uint64_t)i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  index[i] = (int64_t)(z % (uint64_t)n);
}

}  // namespace mlp
}  // namespace bbkde
