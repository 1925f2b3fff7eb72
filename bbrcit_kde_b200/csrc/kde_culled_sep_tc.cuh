// Factored culled sum on 32 x 32 grid tiles with the accumulation on the
// 5th-generation tensor cores (tcgen05, sm_100a).
//
// The culling, the near/far split, the per-slot thresholds and the bound are
// k_pair_sum_culled_sep's (kde_culled_sep.cuh, S = 1). What changes is how a
// summed reference tile reaches the points: per reference j the block computes
// the 32 column factors u_x(q_x,c - x_j) and the 32 row factors m_j u_y(q_y,r -
// y_j), and every point (r, c) needs sum_j Y[r][j] X[c][j] -- a 32 x 32 x 256
// product per reference tile, which the FFMA form feeds from shared memory at 2
// bytes of loads per multiply-add. Here it is a tcgen05.mma chain instead:
//   * each FP32 factor v is split into two TF32 terms, hi = v rounded to TF32
//     and lo = v - hi, of which the tensor core reads the leading 11 bits (hi +
//     lo carries 21 or more of v's 24 bits), and one kind::tf32 MMA of M = 64,
//     N = 64, K = 8 multiplies A = [Y_hi; Y_lo] (rows)
//     by B = [X_hi; X_lo] (columns), so its four 32 x 32 quadrants are the four
//     cross products; a point's value is the sum of its four quadrant entries,
//     the small three first;
//   * K runs over the references of one sub-chunk (32 = four MMAs) into a fresh
//     FP32 accumulator in tensor memory; every thread then reads its points'
//     entries (tcgen05.ld 16x256b) and folds the sub-chunk's sum into its
//     per-point Kahan accumulators, as the FFMA form folds one FP32 partial per
//     32 references;
//   * operands use the canonical K-major layout without swizzle (8-row x 16-byte
//     core matrices; element (m, k) at (k / 4) * 1024 + (m / 8) * 128 + (m % 8) *
//     16 + (k % 4) * 4), double-buffered in shared memory; two 64-column
//     accumulators in tensor memory alternate, so that the MMAs of sub-chunk s run
//     while the block computes the factors of s + 1 and folds s - 1.
// Row order of A: rows 16 q .. 16 q + 15 land in TMEM lane quarter q (the M = 64
// data path uses lanes 0-15 of each quarter), and row 16 q + 8 p + i holds part p
// (hi, lo) of tile row 8 q + i, so that a 16x256b read hands one thread both parts
// of its row. Two block shapes, four blocks per SM either way: NT = 128 threads
// (118 registers), each owning 8 points and making the factors of 4 tile rows or
// columns per group, or NT = 256 (64 registers), each owning 4 points and making 2.
// With 256, warps w and w + 4 share lane quarter w % 4 and split the columns.
// Thread t of warp w owns tile row 8 (w % 4) + t / 4 and columns 8 j + 2 (t % 4) +
// e, j = PP (w / 4) + j', j' < PP = 512 / NT, e < 2. The shapes compute the same
// values bitwise; 256 threads hide more latency, which is what a short list of
// tiles (under ~2 waves) needs, while 128 threads run long lists faster.
//
// Accuracy: the split leaves less than 2^-21 of each factor; the MMA chain's FP32
// accumulation over 32 references was measured at up to 6e-7 relative (mean 2e-7)
// against FP64 of the same FP32 factors. The automatic setting uses this kernel
// only for culled sums whose tolerance is at least kSepTcMinRel.
//
// Every wait on an mbarrier is bounded; on expiry the kernel stops issuing work,
// sets *status and writes no results.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kde_culled_sep.cuh"
#include "tc_util.cuh"

namespace bbkde {

constexpr double kSepTcMinRel = 1e-5;   // smallest tolerance the tensor-core form serves
// Resident blocks per SM (all 512 tensor-memory columns), and the list length in
// waves of them from which 128-thread blocks are used instead of 256-thread ones
// (measured on the 8192^2 grid of 4M references at 1e-5: 65,536 tiles 236 ms with
// 128 threads, 258 ms with 256, 282 ms on the FP32 pipe; on the 1025^2 lattice of
// that grid's pipeline, 1,089 tiles in 1.8 waves, the pipeline step 8.25 ms with
// 128 threads, 8.06 ms with 256, 8.27 ms on the FP32 pipe).
constexpr int kSepTcResident = 4;
constexpr int kSepTcMinWaves = 16;
constexpr int kSepTcLongThreads = 128;   // block shape for long tile lists
constexpr int kSepTcShortThreads = 256;  // block shape for short ones
constexpr int kSepTcSub = 32;            // references per accumulator (MMA K)
constexpr int kSepTcOpBytes = 64 * kSepTcSub * 4;   // one 64-row TF32 operand
constexpr uint32_t kSepTcTmemCols = 128;            // two 64-column accumulators
// TF32 x TF32 -> FP32, A and B K-major, N = 64 (bits 17..22: N / 8), M = 64 (bits
// 24..28: M / 16); c_format F32 = 1 at bit 4, a/b_format TF32 = 2 at bits 7, 10.
constexpr uint32_t kSepTcIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((64u >> 4) << 24);
// Dynamic shared memory each block requests beyond its static arrays (about 44
// KB): four blocks (4 x 128 TMEM columns = all 512) fit in an SM's shared memory,
// a fifth does not (nor in its registers), so no block ever waits for tensor
// memory.
constexpr int kSepTcPadBytes = 4 * 1024;

__device__ __forceinline__ uint32_t sep_tc_off(int m, int k) {
  return (uint32_t)((k >> 2) * 1024 + (m >> 3) * 128 + (m & 7) * 16 + (k & 3) * 4);
}

// K-major, no swizzle: leading byte offset (K direction) 1024 B, stride byte
// offset (M/N direction) 128 B, descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t sep_tc_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(1024u >> 4) << 16) |
         ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void sep_tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                           uint32_t accumulate) {
  const uint32_t zero = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kSepTcIdesc), "r"(accumulate), "r"(zero));
}

// Veltkamp split at 11 significant bits (TF32's 10 explicit + the implicit one):
// with c = (2^13 + 1) v, hi = c - (c - v) is v rounded to 11 bits, an exact TF32
// value, and lo = v - hi is exact in FP32 (at most 13 significant bits, |lo| <=
// 2^-11 |v|). The tensor core reads lo's leading 11 bits (a TF32 operand takes
// an FP32 word's sign, exponent and top 10 mantissa bits), so v = hi + lo' + d
// with |d| < 2^-10 |lo| <= 2^-21 |v|. All on the FP32 pipe, two lanes per packed
// instruction (a conversion instruction per term would run at the conversion
// rate, a quarter of MUFU's). a - b is written fma(b, -1, a): exact negation,
// one rounding.
__device__ __forceinline__ void tf32_split2(float2 v, float2 &hi, float2 &lo) {
  const float2 c = __fmul2_rn(v, f2(8193.0f));
  hi = __ffma2_rn(__ffma2_rn(v, f2(-1.0f), c), f2(-1.0f), c);
  lo = __ffma2_rn(hi, f2(-1.0f), v);
}

// 16 lanes x 8 X columns: r[4 j + e] = (lane t / 4, column 8 j + 2 (t % 4) + e),
// r[4 j + 2 + e] = (lane 8 + t / 4, the same column), j < X.
template <int X>
__device__ __forceinline__ void sep_tc_ld(uint32_t taddr, float (&v)[4 * X]) {
  static_assert(X == 2 || X == 4, "16x256b.x2 or .x4");
  uint32_t r[4 * X];
  if constexpr (X == 2) {
    asm volatile("tcgen05.ld.sync.aligned.16x256b.x2.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
  } else {
    asm volatile(
        "tcgen05.ld.sync.aligned.16x256b.x4.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
  }
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 4 * X; ++i) v[i] = __uint_as_float(r[i]);
}

template <int OP, int NT>
__global__ void __launch_bounds__(NT, 4) k_pair_sum_culled_sep_tc(CullArgs a) {
  static_assert(NT == 128 || NT == 256, "block shape");
  constexpr int T = 32;
  constexpr int BLOCK = NT;
  constexpr int PP = 512 / NT;                 // point pairs per thread (and factor rows)
  constexpr int NW = BLOCK / 32;
  constexpr int NS = 8;                        // slots: strips of T / 8 rows
  constexpr int SPR = T / NS;                  // rows per slot
  constexpr int NSUB = kRefTile / kSepTcSub;   // accumulators per reference tile
  constexpr int STG = kRefTile + 4;            // staged column stride
  constexpr bool kGauss = op_gauss(OP);
  constexpr bool kExt = op_has_extra(OP);
  static_assert(kRefTile % BLOCK == 0 && kSepTcSub == 32, "shape");
  static_assert((STG * 4) % 16 == 0, "16-byte record loads");
  // Two operand buffers, each A (64 x 32 TF32) then B (64 x 32 TF32).
  __shared__ __align__(1024) unsigned char s_op[2][2 * kSepTcOpBytes];
  __shared__ __align__(16) float s_c[2 * STG];     // -x | -y of the staged references
  __shared__ __align__(16) float s_s[2 * STG];     // x scale | y scale
  __shared__ __align__(16) float s_m[2 * STG];     // 1 | mass
  __shared__ float s_qx[T], s_qy[T];
  __shared__ int s_list[cull_list_len(BLOCK)];
  __shared__ int s_glist[cull_groups_per_batch(BLOCK)];
  __shared__ int s_wc[NW];
  __shared__ float s_box[NS][4];
  __shared__ float s_th[NS];
  __shared__ unsigned s_min[NS];
  __shared__ float s_red[NW];
  __shared__ double s_d[NS][NW];
  __shared__ double s_b[NS];
  __shared__ __align__(8) uint64_t s_bar[2];       // one per accumulator
  __shared__ uint32_t s_tmem;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const CullQueries &q = a.q;
  const int t = q.tile_list[blockIdx.x];
  const int64_t i0 = (int64_t)(t % q.ntx) * T, j0 = (int64_t)(t / q.ntx) * T;
  if (tid < T) {
    s_qx[tid] = grid_coord(q.gx0, q.gdx, i0 + tid);
    s_qy[tid] = grid_coord(q.gy0, q.gdy, j0 + tid);
  }
  for (int i = tid; i < kRefTile; i += BLOCK) s_m[i] = 1.0f;
  if (tid < NS) {
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
  if (tid < 2)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_bar[tid])));
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&s_tmem)), "r"(kSepTcTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t op_s = smem_u32(&s_op[0][0]);
  const uint32_t bar_s = smem_u32(&s_bar[0]);

  float qx0 = 3e38f, qx1 = -3e38f, qy0 = 3e38f, qy1 = -3e38f;
#pragma unroll
  for (int k = 0; k < NS; ++k) {
    qx0 = fminf(qx0, s_box[k][0]); qx1 = fmaxf(qx1, s_box[k][1]);
    qy0 = fminf(qy0, s_box[k][2]); qy1 = fmaxf(qy1, s_box[k][3]);
  }

  // This thread's points: row 8 warp + lane / 4, columns 8 j + 2 (lane % 4) + e
  // (point k = 2 j + e), with Kahan accumulators.
  // Warp w reads the TMEM lanes of quarter w % 4 and the column half w / 4: its
  // thread t owns tile row 8 (w % 4) + t / 4 and the 4 columns 8 j + 2 (t % 4) + e
  // with j = PP (w / 4) + (k / 2), e = k % 2 (point k < 2 PP).
  const int lq = warp & 3, ch = warp >> 2;
  const int prow = 8 * lq + (lane >> 2);
  auto pcol = [&](int k) { return 8 * (PP * ch + (k >> 1)) + 2 * (lane & 3) + (k & 1); };
  float2 sum[PP], comp[PP];   // points (2 j', 2 j' + 1) per pair
#pragma unroll
  for (int j = 0; j < PP; ++j) { sum[j] = f2(0.f); comp[j] = f2(0.f); }
  auto valid = [&](int k) { return i0 + pcol(k) < q.gnx && j0 + prow < q.gny; };

  // This thread's factors: references 4 kg .. 4 kg + 3 of a sub-chunk, of the
  // tile rows (half 0: A, with the mass) or columns (half 1: B) r8 + 8 i, i = PP rs
  // + i', i' < PP.
  const int kg = (tid >> 4) & 7, half = (tid >> 3) & 1, r8 = tid & 7, rs = tid >> 7;
  float fq[PP];
  uint32_t o_hi[PP], o_lo[PP];   // byte offsets in a buffer of the hi and lo rows
#pragma unroll
  for (int ii = 0; ii < PP; ++ii) {
    const int i = PP * rs + ii;
    fq[ii] = half ? s_qx[r8 + 8 * i] : s_qy[r8 + 8 * i];
    const int mh = half ? r8 + 8 * i : 16 * i + r8;
    const int ml = half ? 32 + r8 + 8 * i : 16 * i + 8 + r8;
    o_hi[ii] = (uint32_t)(half * kSepTcOpBytes) + sep_tc_off(mh, 4 * kg);
    o_lo[ii] = (uint32_t)(half * kSepTcOpBytes) + sep_tc_off(ml, 4 * kg);
  }
  const int foff = half ? 0 : STG;

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

  // Accumulator pipeline. Group g (one sub-chunk of 32 references) is written by
  // factor() into operand buffer g % 2, multiplied by four MMAs into accumulator
  // g % 2 and committed to mbarrier g % 2 (its (g / 2)-th phase); it is folded in
  // the next step, after group g + 1 has been issued. A barrier's next phase is
  // only committed after every thread has waited for its previous one, so that no
  // phase completes unobserved.
  uint32_t g_next = 0, g_done = 0;   // groups issued, groups folded
  bool my_fail = false, failed = false;

  auto factor = [&](int b, int sub) {
    const int j = foff + sub + 4 * kg;
    const float4 c4 = *reinterpret_cast<const float4 *>(&s_c[j]);
    const float4 s4 = *reinterpret_cast<const float4 *>(&s_s[j]);
    const float4 m4 = *reinterpret_cast<const float4 *>(&s_m[j]);
    const float2 ca = make_float2(c4.x, c4.y), cb = make_float2(c4.z, c4.w);
    const float2 sa = make_float2(s4.x, s4.y), sb = make_float2(s4.z, s4.w);
    const float2 ma = make_float2(m4.x, m4.y), mb = make_float2(m4.z, m4.w);
    unsigned char *base = &s_op[b][0];
#pragma unroll
    for (int i = 0; i < PP; ++i) {
      const float2 da = __fadd2_rn(f2(fq[i]), ca), db = __fadd2_rn(f2(fq[i]), cb);
      const float2 dda = __fmul2_rn(da, da), ddb = __fmul2_rn(db, db);
      float2 ua, ub;
      if (kGauss) {
        const float2 ea = __fmul2_rn(sa, dda), eb = __fmul2_rn(sb, ddb);
        ua = make_float2(ex2_approx(ea.x), ex2_approx(ea.y));
        ub = make_float2(ex2_approx(eb.x), ex2_approx(eb.y));
      } else {
        ua = __ffma2_rn(sa, dda, f2(1.0f));
        ub = __ffma2_rn(sb, ddb, f2(1.0f));
        ua = make_float2(fmaxf(ua.x, 0.f), fmaxf(ua.y, 0.f));
        ub = make_float2(fmaxf(ub.x, 0.f), fmaxf(ub.y, 0.f));
      }
      const float2 va = __fmul2_rn(ma, ua), vb = __fmul2_rn(mb, ub);
      float2 ha, la, hb, lb;
      tf32_split2(va, ha, la);
      tf32_split2(vb, hb, lb);
      *reinterpret_cast<float4 *>(base + o_hi[i]) = make_float4(ha.x, ha.y, hb.x, hb.y);
      *reinterpret_cast<float4 *>(base + o_lo[i]) = make_float4(la.x, la.y, lb.x, lb.y);
    }
  };

  // Fold accumulator b (every thread, after its group's wait) into the points.
  auto fold = [&](int b) {
    // columns of X_hi (8 PP ch ..) and of X_lo (32 + 8 PP ch ..) of this warp
    float v[4 * PP], w[4 * PP];
    const uint32_t ta =
        tmem + (uint32_t)(b * 64 + 8 * PP * ch) + ((uint32_t)(lq * 32) << 16);
    sep_tc_ld<PP>(ta, v);
    sep_tc_ld<PP>(ta + 32u, w);
    const float2 m1 = f2(-1.0f);
#pragma unroll
    for (int j = 0; j < PP; ++j) {
      // quadrants of points (2 j, 2 j + 1): lo.hi, hi.lo, lo.lo first, then hi.hi
      const float2 hh = make_float2(v[4 * j], v[4 * j + 1]);
      const float2 lh = make_float2(v[4 * j + 2], v[4 * j + 3]);
      const float2 hl = make_float2(w[4 * j], w[4 * j + 1]);
      const float2 ll = make_float2(w[4 * j + 2], w[4 * j + 3]);
      const float2 x = __fadd2_rn(__fadd2_rn(__fadd2_rn(lh, hl), ll), hh);
      // Kahan, a - b as fma(b, -1, a): exact negation, one rounding
      const float2 y = __ffma2_rn(comp[j], m1, x);
      const float2 t2 = __fadd2_rn(sum[j], y);
      comp[j] = __ffma2_rn(y, m1, __ffma2_rn(sum[j], m1, t2));
      sum[j] = t2;
    }
  };

  // Wait for group g and fold it.
  auto retire = [&](uint32_t g) {
    if (!tc_wait(bar_s + 8u * (g & 1u), (g >> 1) & 1u)) my_fail = true;
    tc_fence_after();
    if (!my_fail) fold((int)(g & 1u));
  };

  // One sub-chunk: factors into buffer g % 2, MMAs of group g, fold of g - 1.
  auto sub_step = [&](int sub) {
    const uint32_t g = g_next;
    const int b = (int)(g & 1u);
    factor(b, sub);
    fence_async_smem();
    tc_fence_before();
    failed = __syncthreads_or(my_fail) != 0;
    if (failed) return;
    if (tid == 0) {
      tc_fence_after();
      const uint32_t as = op_s + (uint32_t)(b * 2 * kSepTcOpBytes), bs = as + kSepTcOpBytes;
#pragma unroll
      for (int s = 0; s < kSepTcSub / 8; ++s)
        sep_tc_mma(tmem + (uint32_t)(b * 64), sep_tc_desc(as + s * 2048),
                   sep_tc_desc(bs + s * 2048), s > 0 ? 1u : 0u);
      tc_commit(bar_s + 8u * (uint32_t)b);
    }
    g_next = g + 1;
    if (g_done < g) {
      retire(g - 1);
      g_done = g;
    }
  };

  // Fold the last issued group (pass boundaries); every thread agrees on failure.
  auto drain = [&]() {
    if (!failed && g_done < g_next) {
      retire(g_next - 1);
      g_done = g_next;
    }
    tc_fence_before();
    failed = __syncthreads_or(my_fail) != 0;
  };

  // Sum the references [t0, t1) of one tile into the points' accumulators.
  auto sum_tile = [&](int64_t t0, int64_t t1) {
    if (failed) return;
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
    for (int sb = 0; sb < NSUB && !failed; ++sb) sub_step(sb * kSepTcSub);
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
        [&](const RefTile &rt) { return needed(rt, phase, false); }, sum_list);
    drain();
  };

  auto point_sum = [&](int k) {
    return (k & 1) ? sum[k >> 1].y - comp[k >> 1].y : sum[k >> 1].x - comp[k >> 1].x;
  };
  double smin_all = 0.0, ratio = 0.0;
  if (kGauss) {
    pass(1);   // near field
    if (!failed) {
      float mn = INFINITY;
#pragma unroll
      for (int k = 0; k < 2 * PP; ++k)
        if (valid(k)) mn = fminf(mn, fmaxf(point_sum(k), 0.f));
      if (mn < INFINITY) atomicMin(&s_min[prow / SPR], __float_as_uint(mn));
    }
    __syncthreads();
    if (tid < NS) {
      const double mk = (double)__uint_as_float(s_min[tid]);
      const double allow = fmax(a.rel * mk, a.abs_n);
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
      double bsum = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) bsum += s_d[tid][w];
      s_b[tid] = bsum;
    }
    __syncthreads();
    smin_all = INFINITY;
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      const double mk = (double)__uint_as_float(s_min[k]);
      smin_all = fmin(smin_all, mk);
      if (s_b[k] > 0.0)
        ratio = fmax(ratio, s_b[k] * exp2((double)s_th[k]) / fmax(a.rel * mk, a.abs_n));
    }
  } else {
    pass(0);
  }
  if (tid == 0) {
    a.blk_bound[blockIdx.x] = failed ? INFINITY : ratio;
    a.blk_smin[blockIdx.x] = smin_all;
    a.blk_tiles[blockIdx.x] = summed;
    if (failed && a.status) atomicExch(a.status, 1);
  }
  if (!failed) {
#pragma unroll
    for (int k = 0; k < 2 * PP; ++k) {
      if (!valid(k)) continue;
      q.out[(j0 + prow) * q.gnx + (i0 + pcol(k))] =
          q.scale * ((k & 1) ? (double)sum[k >> 1].y - (double)comp[k >> 1].y
                             : (double)sum[k >> 1].x - (double)comp[k >> 1].x);
    }
  }
  // Every issued group has been waited for; after an expired wait, wait (bounded)
  // once more for the last issued group, which completes after all earlier ones.
  if (failed && g_next > 0) tc_wait(bar_s + 8u * ((g_next - 1) & 1u), ((g_next - 1) >> 1) & 1u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kSepTcTmemCols));
}

}  // namespace bbkde
