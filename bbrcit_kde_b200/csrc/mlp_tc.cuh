// Surrogate inference on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Same network and arithmetic as k_mlp_infer (mlp.cuh): FP32 input layer,
// two 128 x 128 BF16 layers with FP32 accumulation, FP32 output layer, SiLU.
// Here the 128 x 128 layers are single tcgen05.mma instructions
// (M = 128 points, N = 128 features, K = 16 per instruction, 8 per layer; 16 with
// two-term activations) reading both operands from shared memory and
// accumulating in tensor memory:
//   * one CTA per SM, two warpgroups; each warpgroup owns a 128-point tile, a
//     128-column FP32 accumulator in TMEM and an mbarrier, and the two share the
//     BF16 weight matrices staged once in shared memory, so one warpgroup's
//     epilogue (bias, SiLU, BF16 packing) overlaps the other's MMAs;
//   * thread t of a warpgroup owns point t of its tile: it computes the input
//     layer, writes its activation row into the A operand, and after the MMA
//     reads its accumulator row back from TMEM lane t (tcgen05.ld 32x32b);
//   * operands use the canonical K-major layout without swizzle: element (r, k)
//     of a 128 x 128 BF16 matrix at byte (k / 8) * 2048 + (r / 8) * 128 +
//     (r % 8) * 16 + (k % 8) * 2, i.e. 8 x 16-byte core matrices, 128 B apart
//     along rows (stride byte offset) and 2048 B apart along K (leading byte
//     offset);
//   * every wait on an mbarrier is bounded; on expiry the kernel records an
//     error in *status and stops issuing work.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "mlp.cuh"
#include "tc_util.cuh"

namespace bbkde {
namespace mlp {

constexpr int kTcRows = 128;                 // points per tile (MMA M)
constexpr int kTcWarpgroups = 2;             // tiles in flight per CTA
constexpr int kTcThreads = 128 * kTcWarpgroups;
constexpr uint32_t kTcTmemCols = 128 * kTcWarpgroups;
constexpr uint32_t kTcMatBytes = 128 * 128 * 2;   // one 128 x 128 BF16 operand
// BF16 x BF16 -> FP32, A and B K-major, N = 128 (bits 17..22: N / 8), M = 128
// (bits 24..28: M / 16); c_format F32 = 1 at bit 4, a/b_format BF16 = 1 at bits 7, 10.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) |
                              ((128u >> 4) << 24);

template <bool kSplit>
struct TcSmem {
  static constexpr size_t kW = 0;                                  // W2, W3
  static constexpr size_t kA = 2 * kTcMatBytes;                    // per warpgroup: hi (, lo)
  static constexpr size_t kAPerWg = (kSplit ? 2 : 1) * kTcMatBytes;
  static constexpr size_t kF = kA + kTcWarpgroups * kAPerWg;       // FP32 vectors
  static constexpr size_t kFloats = 2 * kH + 3 * kH + kH;          // W1, b1..b3, w4
  static constexpr size_t kBar = kF + kFloats * sizeof(float);     // mbarriers (8 B each)
  static constexpr size_t kTmem = kBar + 8 * kTcWarpgroups;        // TMEM base address
  static constexpr size_t kFail = kTmem + 8;                       // per warpgroup: wait expired
  static constexpr size_t kBytes = kFail + 4 * kTcWarpgroups;
};

__device__ __forceinline__ uint32_t tc_off(int r, int k) {
  return (uint32_t)((k >> 3) * 2048 + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor: K-major, no swizzle, LBO 2048 B, SBO 128 B,
// descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(2048u >> 4) << 16) |
         ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
}

// The same stored matrix read transposed, as an MN-major operand: a matrix
// stored at tc_off(r, k) has its second index k contiguous in 16-byte runs, so
// read with k as the M (or N) dimension and r as K it is the canonical MN-major
// layout without swizzle, whose K-direction core-matrix stride goes in the
// leading byte offset (128 B between groups of 8 r) and the M/N-direction stride
// in the stride byte offset (2048 B between groups of 8 k). One K = 16 step of
// such an operand advances 2 x 128 B (a K-major one 2 x 2048 B).
__device__ __forceinline__ uint64_t tc_desc_mn(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)(2048u >> 4) << 32) | (1ull << 46);
}
constexpr uint32_t kTcAMajorMN = 1u << 15;   // instruction descriptor: A is MN-major
constexpr uint32_t kTcBMajorMN = 1u << 16;   // B is MN-major

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate, uint32_t idesc = kTcIdesc) {
  const uint32_t zero = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(zero));
}

// D (+)= A x B over K = 128 (8 instructions of K = 16), M = N = 128. A and B are
// stored 128 x 128 BF16 matrices at tc_off; a_mn / b_mn read them transposed.
__device__ __forceinline__ void tc_gemm128(uint32_t tmem_d, uint32_t a, bool a_mn, uint32_t b,
                                           bool b_mn, bool accumulate) {
  const uint32_t idesc = kTcIdesc | (a_mn ? kTcAMajorMN : 0u) | (b_mn ? kTcBMajorMN : 0u);
#pragma unroll
  for (int s = 0; s < kH / 16; ++s) {
    const uint64_t ad = a_mn ? tc_desc_mn(a + s * 256) : tc_desc(a + s * 4096);
    const uint64_t bd = b_mn ? tc_desc_mn(b + s * 256) : tc_desc(b + s * 4096);
    tc_mma(tmem_d, ad, bd, (accumulate || s > 0) ? 1u : 0u, idesc);
  }
}

__device__ __forceinline__ void wg_sync(int wg) {
  asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Eight activations (features k0 .. k0 + 7 of row r) into the A operand(s).
template <bool kSplit>
__device__ __forceinline__ void tc_store8(unsigned char *ahi, unsigned char *alo, int r, int k0,
                                          const float *a) {
  uint32_t hi[4], lo[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a[2 * i], a[2 * i + 1]);
    hi[i] = *reinterpret_cast<const uint32_t *>(&h);
    if (kSplit) {
      const float2 hf = __bfloat1622float2(h);
      lo[i] = pack_bf16(a[2 * i] - hf.x, a[2 * i + 1] - hf.y);
    }
  }
  *reinterpret_cast<uint4 *>(ahi + tc_off(r, k0)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  if (kSplit)
    *reinterpret_cast<uint4 *>(alo + tc_off(r, k0)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
}

// The two 128 x 128 BF16 weight matrices (row-major [n][k] in global memory)
// into the canonical layout, 16 bytes (8 consecutive k of one row n) per copy:
// consecutive threads take consecutive rows, so a warp's shared-memory stores
// fill 512 contiguous bytes.
__device__ __forceinline__ void tc_stage_weights(unsigned char *W2, unsigned char *W3,
                                                 const __nv_bfloat16 *w2,
                                                 const __nv_bfloat16 *w3, int tid,
                                                 int nthreads) {
  const uint4 *g2 = reinterpret_cast<const uint4 *>(w2);
  const uint4 *g3 = reinterpret_cast<const uint4 *>(w3);
  for (int i = tid; i < kH * kH / 8; i += nthreads) {
    const int n = i % kH, k0 = (i / kH) * 8;
    const int gi = n * (kH / 8) + k0 / 8;
    *reinterpret_cast<uint4 *>(W2 + tc_off(n, k0)) = __ldg(g2 + gi);
    *reinterpret_cast<uint4 *>(W3 + tc_off(n, k0)) = __ldg(g3 + gi);
  }
}

struct TcArgs {
  InferArgs in;
  int *status;   // set to 1 if a wait expired
};

template <bool kSplit>
__global__ void __launch_bounds__(kTcThreads, 1) k_mlp_infer_tc(TcArgs ta) {
  using L = TcSmem<kSplit>;
  extern __shared__ __align__(16) unsigned char smem[];   // 16 B: no-swizzle operands
  const InferArgs &a = ta.in;
  unsigned char *W2 = smem + L::kW, *W3 = W2 + kTcMatBytes;
  float *fp = reinterpret_cast<float *>(smem + L::kF);
  float *W1 = fp, *b1 = W1 + 2 * kH, *b2 = b1 + kH, *b3 = b2 + kH, *w4 = b3 + kH;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::kBar);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L::kTmem);
  volatile int *fail = reinterpret_cast<volatile int *>(smem + L::kFail);

  const int tid = threadIdx.x, wg = tid >> 7, row = tid & 127, warp = tid >> 5;
  // Weights into the canonical layout; FP32 vectors.
  tc_stage_weights(W2, W3, a.w2, a.w3, tid, kTcThreads);
  for (int i = tid; i < 2 * kH; i += kTcThreads) W1[i] = a.params[kOffW1 + i];
  for (int i = tid; i < kH; i += kTcThreads) {
    b1[i] = a.params[kOffB1 + i];
    b2[i] = a.params[kOffB2 + i];
    b3[i] = a.params[kOffB3 + i];
    w4[i] = a.params[kOffW4 + i];
  }
  if (tid < kTcWarpgroups) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[tid])));
    fail[tid] = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(tmem_slot)), "r"(kTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_async_smem();
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const float b4 = a.params[kOffB4];

  unsigned char *ahi = smem + L::kA + wg * L::kAPerWg;
  unsigned char *alo = ahi + kTcMatBytes;
  const uint32_t tmem_d = tmem + (uint32_t)(wg * 128);          // this warpgroup's columns
  const uint32_t taddr = tmem_d + ((uint32_t)((warp & 3) * 32) << 16);   // this warp's lanes
  const uint32_t mbar = smem_u32(&bars[wg]);
  const uint32_t w2s = smem_u32(W2), w3s = smem_u32(W3);
  const uint32_t ahs = smem_u32(ahi), als = smem_u32(alo);
  uint32_t phase = 0;
  bool ok = true;

  // One 128 x 128 layer: A (and A_lo) x W^T -> TMEM, issued by thread 0 of the
  // warpgroup after every row is written; returns false (uniformly across the
  // warpgroup) if a wait expired.
  auto layer = [&](uint32_t ws) -> bool {
    fence_async_smem();
    tc_fence_before();
    wg_sync(wg);
    if (row == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < kH / 16; ++s) {
        const uint64_t bd = tc_desc(ws + s * 4096);
        if (kSplit) tc_mma(tmem_d, tc_desc(als + s * 4096), bd, s > 0 ? 1u : 0u);
        tc_mma(tmem_d, tc_desc(ahs + s * 4096), bd, (kSplit || s > 0) ? 1u : 0u);
      }
      tc_commit(mbar);
    }
    if (!tc_wait(mbar, phase)) fail[wg] = 1;
    phase ^= 1u;
    tc_fence_after();
    wg_sync(wg);          // every thread of the warpgroup has waited: one verdict
    return fail[wg] == 0;
  };

  const int64_t tiles = (a.n + kTcRows - 1) / kTcRows;
  for (int64_t tile = (int64_t)blockIdx.x * kTcWarpgroups + wg; tile < tiles && ok;
       tile += (int64_t)gridDim.x * kTcWarpgroups) {
    const int64_t p = tile * kTcRows + row;
    float2 q = make_float2(0.f, 0.f);
    if (a.xy) {
      if (p < a.n) q = a.xy[p];
    } else {
      q = make_float2((float)(a.gx0 + (double)(p % a.gnx) * a.gdx),
                      (float)(a.gy0 + (double)(p / a.gnx) * a.gdy));
    }
    const float x = (q.x - a.norm.cx) * a.norm.sx, y = (q.y - a.norm.cy) * a.norm.sy;
    // Input layer (FP32) -> A.
#pragma unroll 1
    for (int k0 = 0; k0 < kH; k0 += 8) {
      float v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int n = k0 + i;
        v[i] = silu(fmaf(W1[2 * n], x, fmaf(W1[2 * n + 1], y, b1[n])));
      }
      tc_store8<kSplit>(ahi, alo, row, k0, v);
    }
    // Hidden layer 2 -> A, hidden layer 3 -> output.
    float out = 0.f;
#pragma unroll 1
    for (int l = 0; l < 2 && ok; ++l) {
      if (!layer(l == 0 ? w2s : w3s)) { ok = false; break; }
      const float *bias = l == 0 ? b2 : b3;
#pragma unroll 1
      for (int c = 0; c < kH; c += 32) {
        float v[32];
        tc_ld32(taddr + (uint32_t)c, v);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = silu(v[i] + bias[c + i]);
        if (l == 0) {
#pragma unroll
          for (int j = 0; j < 32; j += 8) tc_store8<kSplit>(ahi, alo, row, c + j, v + j);
        } else {
#pragma unroll
          for (int i = 0; i < 32; ++i) out = fmaf(w4[c + i], v[i], out);
        }
      }
    }
    if (ok && p < a.n) a.out[p] = a.norm.mu + a.norm.sigma * (out + b4);
  }
  if (!ok && row == 0) atomicExch(ta.status, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcTmemCols));
}

// ===========================================================================
// Training step on tcgen05: forward and backward of 128 points per CTA.
//
// One warpgroup, thread t = point t = TMEM lane t. The four 128 x 128 x 128
// products of a step run on the tensor cores from the same stored BF16
// matrices (canonical K-major at tc_off), reading them transposed (MN-major)
// where the product needs it:
//   forward   Z2 = A1 W2^T, Z3 = A2 W3^T                 (A, B K-major)
//   input     dA2 = dZ3 W3, dA1 = dZ2 W2                  (A K-major, B MN-major)
//   weights   dW3 = dZ3^T A2, dW2 = dZ2^T A1 (K = points) (A, B MN-major)
// TMEM (512 columns): [0, 128) Z2, kept for silu'(z2); [128, 256) Z3, then dA2,
// then dA1; [256, 384) dW3, then dW2. The 2 -> 128 and 128 -> 1 layers and every
// per-feature sum over the points (bias gradients, dW1, dw4) run in FP32 on the
// CUDA cores; the sums are warp butterflies then a fixed-order sum over the four
// warps, so a step is deterministic. Rounding points (the FP64 restatement in
// the tests follows them): A1 = bf16(silu(z1)), A2 = bf16(silu(z2)), dZ3 =
// bf16(dz3), dZ2 = bf16(dz2); z2, z3, dA and dW stay FP32; bias and vector
// gradients sum the FP32 dz. Per CTA the gradient partial is written in the
// parameter layout (k_mlp_reduce sums the partials in a fixed order). Every
// mbarrier wait is bounded; on expiry *status is set and the CTA stops.
// ===========================================================================
constexpr int kTcTrainPts = 128;
constexpr uint32_t kTcTrainCols = 512;

struct TcTrainSmem {
  static constexpr size_t kW2 = 0;
  static constexpr size_t kW3 = kW2 + kTcMatBytes;
  static constexpr size_t kA1 = kW3 + kTcMatBytes;
  static constexpr size_t kA2 = kA1 + kTcMatBytes;
  static constexpr size_t kDZ = kA2 + kTcMatBytes;               // dZ3, then dZ2
  static constexpr size_t kF = kDZ + kTcMatBytes;                // FP32 vectors
  static constexpr size_t kFloats = 2 * kH + 4 * kH + 4 * kH;    // W1, b1 b2 b3 w4, red[4][kH]
  static constexpr size_t kBar = kF + kFloats * sizeof(float);
  static constexpr size_t kTmem = kBar + 8;
  static constexpr size_t kFail = kTmem + 8;
  static constexpr size_t kBytes = kFail + 16;
};

struct TcTrainArgs {
  TrainArgs t;
  int *status;   // set to 1 if a wait expired
};

// Sum over the 32 lanes of a warp, per index: after the call lane j holds
// sum_lanes v[j] in v[0] (butterfly: at offset o a lane keeps the half of its
// window that its bit o selects and adds the partner's copy of it).
__device__ __forceinline__ float warp_transpose_sum(float (&v)[32], int lane) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    const bool up = (lane & o) != 0;
#pragma unroll
    for (int i = 0; i < o; ++i) {
      const float send = up ? v[i] : v[i + o];
      const float keep = up ? v[i + o] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
  return v[0];
}

__global__ void __launch_bounds__(kTcRows, 1) k_mlp_train_tc(TcTrainArgs ta) {
  using L = TcTrainSmem;
  extern __shared__ __align__(16) unsigned char smem[];
  const TrainArgs &a = ta.t;
  unsigned char *W2 = smem + L::kW2, *W3 = smem + L::kW3, *A1 = smem + L::kA1,
                *A2 = smem + L::kA2, *DZ = smem + L::kDZ;
  float *fp = reinterpret_cast<float *>(smem + L::kF);
  float *W1 = fp, *b1 = W1 + 2 * kH, *b2 = b1 + kH, *b3 = b2 + kH, *w4 = b3 + kH;
  float *red = w4 + kH;   // [4 warps][kH]
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L::kBar);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + L::kTmem);
  volatile int *fail = reinterpret_cast<volatile int *>(smem + L::kFail);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  tc_stage_weights(W2, W3, a.w2, a.w3, tid, kTcRows);
  for (int i = tid; i < 2 * kH; i += kTcRows) W1[i] = a.params[kOffW1 + i];
  for (int i = tid; i < kH; i += kTcRows) {
    b1[i] = a.params[kOffB1 + i];
    b2[i] = a.params[kOffB2 + i];
    b3[i] = a.params[kOffB3 + i];
    w4[i] = a.params[kOffW4 + i];
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    fail[0] = 0;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(tmem_slot)), "r"(kTcTrainCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // This thread's point.
  const int64_t p = (int64_t)blockIdx.x * kTcTrainPts + tid;
  const bool valid = p < a.batch;
  float x = 0.f, y = 0.f, target = 0.f;
  if (valid) {
    const int64_t row = a.index[p];
    const float2 q = a.xy[row];
    x = (q.x - a.norm.cx) * a.norm.sx;
    y = (q.y - a.norm.cy) * a.norm.sy;
    target = (a.target[row] - a.norm.mu) / a.norm.sigma;
  }
  fence_async_smem();
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lanes = (uint32_t)(warp * 32) << 16;
  const uint32_t tZ2 = tmem, tZ3 = tmem + 128, tW = tmem + 256;
  const uint32_t mbar = smem_u32(bar);
  const uint32_t sW2 = smem_u32(W2), sW3 = smem_u32(W3), sA1 = smem_u32(A1),
                 sA2 = smem_u32(A2), sDZ = smem_u32(DZ);
  uint32_t phase = 0;
  const float b4 = a.params[kOffB4];
  const float inv_b = 1.0f / (float)a.batch;
  float *gp = a.grad_part + (int64_t)blockIdx.x * kPartStride;

  // Issue the products of `body` from thread 0 once every thread's operand
  // rows are in shared memory; wait for them (bounded). Uniform verdict.
  auto run = [&](auto body) -> bool {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      body();
      tc_commit(mbar);
    }
    if (!tc_wait(mbar, phase)) fail[0] = 1;
    phase ^= 1u;
    tc_fence_after();
    __syncthreads();
    return fail[0] == 0;
  };
  // Per-feature sums over the CTA's points of v (32 features from c0): the warp
  // butterfly, then warp partials summed in warp order by thread c0 + lane.
  auto colsum = [&](float (&v)[32], int c0, float *dst, int stride) {
    const float s = warp_transpose_sum(v, lane);
    red[warp * kH + c0 + lane] = s;
    __syncthreads();
    if (tid < 32) {
      const int n = c0 + tid;
      dst[n * stride] = ((red[n] + red[kH + n]) + red[2 * kH + n]) + red[3 * kH + n];
    }
    __syncthreads();
  };
  bool ok = true;

  // ---- forward -----------------------------------------------------------
#pragma unroll 1
  for (int k0 = 0; k0 < kH; k0 += 8) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int n = k0 + i;
      v[i] = silu(fmaf(W1[2 * n], x, fmaf(W1[2 * n + 1], y, b1[n])));
    }
    tc_store8<false>(A1, nullptr, tid, k0, v);
  }
  ok = run([&] { tc_gemm128(tZ2, sA1, false, sW2, false, false); });
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < kH; c += 32) {
      float v[32];
      tc_ld32(tZ2 + lanes + (uint32_t)c, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) v[i] = silu(v[i] + b2[c + i]);
#pragma unroll
      for (int j = 0; j < 32; j += 8) tc_store8<false>(A2, nullptr, tid, c + j, v + j);
    }
    ok = run([&] { tc_gemm128(tZ3, sA2, false, sW3, false, false); });
  }
  float out = 0.f;
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < kH; c += 32) {
      float v[32];
      tc_ld32(tZ3 + lanes + (uint32_t)c, v);
#pragma unroll
      for (int i = 0; i < 32; ++i) out = fmaf(w4[c + i], silu(v[i] + b3[c + i]), out);
    }
  }
  // ---- output layer and dz3 ----------------------------------------------
  const float e = valid ? out + b4 - target : 0.f;
  const float dy = 2.f * e * inv_b;   // dL/dy
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < kH; c += 32) {
      float z[32], dz[32], aw[32];
      tc_ld32(tZ3 + lanes + (uint32_t)c, z);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const float zz = z[i] + b3[c + i];
        dz[i] = dy * w4[c + i] * silu_grad(zz);
        aw[i] = dy * silu(zz);
      }
#pragma unroll
      for (int j = 0; j < 32; j += 8) tc_store8<false>(DZ, nullptr, tid, c + j, dz + j);
      colsum(dz, c, gp + kOffB3, 1);
      colsum(aw, c, gp + kOffW4, 1);
    }
    // dA2 = dZ3 W3 -> [128, 256); dW3 = dZ3^T A2 -> [256, 384)
    ok = run([&] {
      tc_gemm128(tZ3, sDZ, false, sW3, true, false);
      tc_gemm128(tW, sDZ, true, sA2, true, false);
    });
  }
  // ---- dz2, dW3 ------------------------------------------------------------
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < kH; c += 32) {
      float d[32], z[32];
      tc_ld32(tZ3 + lanes + (uint32_t)c, d);
      tc_ld32(tZ2 + lanes + (uint32_t)c, z);
#pragma unroll
      for (int i = 0; i < 32; ++i) d[i] *= silu_grad(z[i] + b2[c + i]);
#pragma unroll
      for (int j = 0; j < 32; j += 8) tc_store8<false>(DZ, nullptr, tid, c + j, d + j);
      colsum(d, c, gp + kOffB2, 1);
    }
#pragma unroll 1
    for (int c = 0; c < kH; c += 32) {   // row tid of dW3
      float g[32];
      tc_ld32(tW + lanes + (uint32_t)c, g);
      // 16-byte stores: partials are kPartStride floats apart (a multiple of 4)
      float4 *dst = reinterpret_cast<float4 *>(gp + kOffW3 + tid * kH + c);
#pragma unroll
      for (int i = 0; i < 8; ++i)
        dst[i] = make_float4(g[4 * i], g[4 * i + 1], g[4 * i + 2], g[4 * i + 3]);
    }
    // dA1 = dZ2 W2 -> [128, 256); dW2 = dZ2^T A1 -> [256, 384)
    ok = run([&] {
      tc_gemm128(tZ3, sDZ, false, sW2, true, false);
      tc_gemm128(tW, sDZ, true, sA1, true, false);
    });
  }
  // ---- dz1 and the first layer; dW2 --------------------------------------
  if (ok) {
#pragma unroll 1
    for (int c = 0; c < kH; c += 32) {
      float d[32], dxv[32], dyv[32];
      tc_ld32(tZ3 + lanes + (uint32_t)c, d);
#pragma unroll
      for (int i = 0; i < 32; ++i) {
        const int n = c + i;
        d[i] *= silu_grad(fmaf(W1[2 * n], x, fmaf(W1[2 * n + 1], y, b1[n])));
        dxv[i] = d[i] * x;
        dyv[i] = d[i] * y;
      }
      colsum(d, c, gp + kOffB1, 1);
      colsum(dxv, c, gp + kOffW1, 2);       // dW1[n][0]
      colsum(dyv, c, gp + kOffW1 + 1, 2);   // dW1[n][1]
    }
#pragma unroll 1
    for (int c = 0; c < kH; c += 32) {   // row tid of dW2
      float g[32];
      tc_ld32(tW + lanes + (uint32_t)c, g);
      float4 *dst = reinterpret_cast<float4 *>(gp + kOffW2 + tid * kH + c);
#pragma unroll
      for (int i = 0; i < 8; ++i)
        dst[i] = make_float4(g[4 * i], g[4 * i + 1], g[4 * i + 2], g[4 * i + 3]);
    }
  }
  // ---- db4 and the loss: fixed-order sums over the points ---------------
  red[tid] = dy;
  red[kH + tid] = e * e;
  __syncthreads();
  if (tid == 0) {
    float sd = 0.f, se = 0.f;
    for (int i = 0; i < kTcTrainPts; ++i) {
      sd += red[i];
      se += red[kH + i];
    }
    gp[kOffB4] = sd;
    a.loss_part[blockIdx.x] = se * inv_b;
  }
  if (!ok && tid == 0) atomicExch(ta.status, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcTrainCols));
}

}  // namespace mlp
}  // namespace bbkde
