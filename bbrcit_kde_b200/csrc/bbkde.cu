// libbbkde.so: the C ABI declared in include/bbkde.h.
//
// Host code for the B200 direct kernel-density path. A context owns one
// device's buffers and a stream; point sets live in HBM as FP64 SoA columns
// (x, y, mass, abw, weight) and are packed on the device into per-kernel
// records (kde_device.cuh) only when the kernel, bandwidth or attributes change.
// Every call validates its arguments the way the reference does
// (CudaDirectKde.h:181-190), surfaces every CUDA error as BBKDE_CUDA_ERROR, and
// synchronises its stream before returning.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include "../../include/bbkde.h"
#include "kde_device.cuh"
#include "kde_cv_batch.cuh"
#include "kde_culled.cuh"
#include "kde_culled_sep.cuh"
#include "kde_culled_sep_tc.cuh"
#include "kde_grid.cuh"

using namespace bbkde;

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

struct PointSet {
  int dim = 0;
  int64_t n = 0;
  DevBuf x, y, mass, abw, weight;   // double columns
  uint64_t coord_version = 0;       // bumps on upload
  uint64_t attr_version = 0;        // bumps when mass / abw change
};

// Resolved kernel: device operator, record scales and normalisation.
struct Resolved {
  int op = 0, dim = 0;
  double h1 = 1, h2 = 1;
  double c1_f32 = 0, c2_f32 = 0;   // log2-based scale numerators (FP32 records)
  double c1_f64 = 0, c2_f64 = 0;   // natural-log scale numerators (FP64 records)
  double mass_scale = 1.0;
  double norm = 1.0;               // C(h), reference formulas, FP64
};

struct PackKey {
  int op = -1, dim = 0;
  double h1 = 0, h2 = 0, c1 = 0, c2 = 0, ms = 0;
  uint64_t coord_version = ~0ull, attr_version = ~0ull;
  bool operator==(const PackKey &o) const {
    return op == o.op && dim == o.dim && h1 == o.h1 && h2 == o.h2 && c1 == o.c1 &&
           c2 == o.c2 && ms == o.ms && coord_version == o.coord_version &&
           attr_version == o.attr_version;
  }
};

struct PackCache {
  PackKey key;
  DevBuf rec, ext;
};

// Morton-sorted FP32 records of the reference set and their culling tiles,
// valid for the packed records with the same key.
struct CullCache {
  PackKey key;
  DevBuf rec, ext, tiles, groups;
  int n_tiles = 0;
  int n_groups = 0;
};

struct QueryCache {
  int set = -1;
  uint64_t coord_version = ~0ull;
  DevBuf x, y;
};

constexpr double kLog2e = 1.4426950408889634074;

}  // namespace

struct bbkde_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  PointSet sets[2];
  PackCache pack32, pack64;
  QueryCache q32[2];          // FP32 query coordinates, one slot per point set
  DevBuf partial, out_dev, block_sums, scalars, staging, status;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  double last_ms = 0, last_pairs = 0;
  int64_t last_launches = 0;
  int64_t launch_total = 0;   // every kernel this context has launched
  int forced_variant = -1;    // -1: autotune
  int last_variant = -1;
  // autotuner cache: (op, dim, exclude_self, log2 refs, log2 queries) -> variant
  std::map<std::tuple<int, int, int, int, int>, int> tuned;
  // batched cross-validation buffers and the captured launch graph
  DevBuf cv_x, cv_y, cv_w, cv_cells, cv_sets, cv_items, cv_counter, cv_h, cv_lut,
      cv_part, cv_hist, cv_out, cv_parts;
  cudaGraphExec_t cv_graph = nullptr;
  std::vector<uint64_t> cv_graph_key;
  int64_t cv_counts[2] = {0, 0};   // in-support pairs of the last batched CV launch
  int cv_forced_plan = -1;         // -1: autotune the batched CV work-item plan
  int cv_last_plan = -1;
  // per problem class: device ms of each plan tried so far (< 0: not yet tried)
  std::map<std::tuple<int, int, int, int, int>, std::vector<double>> cv_tuned;
  // culled evaluation: sorted references, sort scratch, sorted queries, per-block
  // bounds; dense-grid pipeline buffers
  CullCache cull;
  DevBuf ms_keys, ms_keys2, ms_perm, ms_perm2, ms_box, ms_tmp, cq_x, cq_y, cq_out, cb_bound,
      cb_smin, cb_tiles, cb_stats, cb_key, cb_key2, cb_sched;
  DevBuf gr_pred, gr_order, gr_tmin, gr_tmax, gr_bad, gr_terr, gr_flag, gr_flag_ord, gr_list,
      gr_nsel, gr_counts, gr_gmax, gr_lat_order, gr_lat_exact, gr_lat_net, gr_q_order, gr_q_exact,
      gr_q_net, gr_resid, gr_cand_ord, gr_cand_xy, gr_cand_net, gr_out, gr_part, gr_rl_idx,
      gr_rl_xy, gr_rl_net;
  cudaEvent_t ev3 = nullptr;
  // smallest positive abw of the reference set, for the (coordinate, attribute)
  // versions it was computed at
  double abw_min = 1.0;
  uint64_t abw_min_cv = ~0ull, abw_min_av = ~0ull;
  std::string err;
};

namespace {

int fail(bbkde_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

#define CUDA_TRY(ctx, call)                                                          \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      return fail(ctx, BBKDE_CUDA_ERROR, std::string(#call) + ": " +               \
                                             cudaGetErrorString(e_));                \
    }                                                                                \
  } while (0)

int ensure(bbkde_ctx *c, DevBuf &b, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (b.cap >= bytes) return BBKDE_OK;
  if (b.p) {
    cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
  }
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(c, BBKDE_ALLOC_FAILED,
                "cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
  }
  b.cap = bytes;
  return BBKDE_OK;
}

void release(DevBuf &b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

#define TRY(expr)                 \
  do {                            \
    int rc_ = (expr);             \
    if (rc_ != BBKDE_OK) return rc_; \
  } while (0)

#define COUNT_LAUNCH(c) (++(c)->launch_total)

inline unsigned grid1d(int64_t n, int block = 256) {
  return (unsigned)std::max<int64_t>(1, (n + block - 1) / block);
}

// Normalisation C(h) exactly as the reference computes it
// (include/Kernels/KernelTraits.h; line numbers in oracle/kde_oracle.c).
double normalization(int kind, int dim, const double *h) {
  switch (kind) {
    case BBKDE_GAUSSIAN:
      if (dim == 1) return 0.3989422804014326779 / (double)(float)h[0];  // float h, :143
      return 0.1591549430918953357 / (h[0] * h[0]);
    case BBKDE_EPANECHNIKOV:
      if (dim == 1) return 0.75 / h[0];
      return 0.6366197723675813431 / (h[0] * h[0]);
    case BBKDE_GAUSSIAN_PRODUCT_2D: return 0.1591549430918953357 / (h[0] * h[1]);
    case BBKDE_EPANECHNIKOV_PRODUCT_2D: return 0.5625 / (h[0] * h[1]);
    case BBKDE_GAUSSIAN_PRODUCT_CONV_2D: return 0.0795774715459476678 / (h[0] * h[1]);
    case BBKDE_EPANECHNIKOV_PRODUCT_CONV_2D: return 0.36 / (h[0] * h[1]);
    case BBKDE_GAUSSIAN_CONV_1D: return 0.2820947917738781434 / h[0];
    case BBKDE_EPANECHNIKOV_CONV_1D: return 0.6 / h[0];
  }
  return 0.0;
}

int resolve(bbkde_ctx *c, const bbkde_kernel_desc *k, Resolved &r) {
  if (!k) return fail(c, BBKDE_INVALID_ARGUMENT, "kernel descriptor is NULL");
  if (k->dim != 1 && k->dim != 2)
    return fail(c, BBKDE_INVALID_ARGUMENT, "kernel dim must be 1 or 2");
  const bool product = k->kind == BBKDE_GAUSSIAN_PRODUCT_2D ||
                       k->kind == BBKDE_EPANECHNIKOV_PRODUCT_2D ||
                       k->kind == BBKDE_GAUSSIAN_PRODUCT_CONV_2D ||
                       k->kind == BBKDE_EPANECHNIKOV_PRODUCT_CONV_2D;
  const bool one_d = k->kind == BBKDE_GAUSSIAN_CONV_1D || k->kind == BBKDE_EPANECHNIKOV_CONV_1D;
  if (k->kind < 0 || k->kind > BBKDE_EPANECHNIKOV_CONV_1D)
    return fail(c, BBKDE_INVALID_ARGUMENT, "unknown kernel kind");
  if (product && k->dim != 2)
    return fail(c, BBKDE_INVALID_ARGUMENT, "product kernels are 2-D");
  if (one_d && k->dim != 1)
    return fail(c, BBKDE_INVALID_ARGUMENT, "1-D convolution kernels need dim 1");
  const double hx = k->h[0], hy = product ? k->h[1] : k->h[0];
  if (!(hx > 0) || !(hy > 0) || !std::isfinite(hx) || !std::isfinite(hy))
    return fail(c, BBKDE_INVALID_ARGUMENT, "bandwidths must be positive and finite");
  r = Resolved();
  r.dim = k->dim;
  r.h1 = hx;
  r.h2 = hy;
  r.norm = normalization(k->kind, k->dim, k->h);
  double g = -0.5;  // exponent factor of the Gaussian family
  switch (k->kind) {
    case BBKDE_GAUSSIAN:
    case BBKDE_GAUSSIAN_PRODUCT_2D:
      break;
    case BBKDE_GAUSSIAN_CONV_1D:
      g = -0.25;
      break;
    case BBKDE_GAUSSIAN_PRODUCT_CONV_2D:
      g = (k->flags & BBKDE_FLAG_EXACT_GAUSS_CONV) ? -0.25 : -0.5;
      break;
    default:
      g = 0.0;
  }
  switch (k->kind) {
    case BBKDE_GAUSSIAN:
    case BBKDE_GAUSSIAN_CONV_1D:
    case BBKDE_GAUSSIAN_PRODUCT_2D:
    case BBKDE_GAUSSIAN_PRODUCT_CONV_2D:
      // (dx^2/hx^2 + dy^2/hy^2) with hx == hy is the isotropic form.
      r.op = (hx == hy) ? OP_GAUSS_ISO : OP_GAUSS_PROD;
      r.c1_f32 = r.c2_f32 = g * kLog2e;
      r.c1_f64 = r.c2_f64 = g;
      break;
    case BBKDE_EPANECHNIKOV:
      r.op = OP_EPAN_ISO;
      r.c1_f32 = r.c2_f32 = r.c1_f64 = r.c2_f64 = -1.0;
      break;
    case BBKDE_EPANECHNIKOV_PRODUCT_2D:
      r.op = OP_EPAN_PROD;
      r.c1_f32 = r.c2_f32 = r.c1_f64 = r.c2_f64 = -1.0;
      break;
    case BBKDE_EPANECHNIKOV_PRODUCT_CONV_2D:
      r.op = OP_EPAN_CONV;
      r.mass_scale = 1.0 / 1024.0;  // 0.03125 per dimension
      break;
    case BBKDE_EPANECHNIKOV_CONV_1D:
      r.op = OP_EPAN_CONV;
      r.mass_scale = 1.0 / 32.0;
      break;
  }
  if (k->dim == 1 && r.op == OP_GAUSS_PROD) r.op = OP_GAUSS_ISO;
  return BBKDE_OK;
}

int check_ctx(bbkde_ctx *c) {
  if (!c) return BBKDE_INVALID_ARGUMENT;
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return fail(c, BBKDE_CUDA_ERROR, cudaGetErrorString(e));
  return BBKDE_OK;
}

// Pack the REFERENCE set into records for `r` (cached).
int ensure_pack(bbkde_ctx *c, const Resolved &r, bool f64) {
  PointSet &s = c->sets[BBKDE_REFERENCE];
  PackCache &pc = f64 ? c->pack64 : c->pack32;
  PackKey key;
  key.op = r.op;
  key.dim = r.dim;
  key.h1 = r.h1;
  key.h2 = r.h2;
  key.c1 = f64 ? r.c1_f64 : r.c1_f32;
  key.c2 = f64 ? r.c2_f64 : r.c2_f32;
  key.ms = r.mass_scale;
  key.coord_version = s.coord_version;
  key.attr_version = s.attr_version;
  if (pc.key == key) return BBKDE_OK;
  const int64_t n = std::max<int64_t>(s.n, 1);
  TRY(ensure(c, pc.rec, (size_t)n * (f64 ? sizeof(double4) : sizeof(float4))));
  TRY(ensure(c, pc.ext, (size_t)n * (f64 ? sizeof(double) : sizeof(float))));
  if (s.n > 0) {
    PackArgs p;
    p.x = s.x.as<double>();
    p.y = s.y.as<double>();
    p.mass = s.mass.as<double>();
    p.abw = s.abw.as<double>();
    p.n = s.n;
    p.op = r.op;
    p.dim = r.dim;
    p.c1 = key.c1;
    p.c2 = key.c2;
    p.h1 = r.h1;
    p.h2 = r.h2;
    p.mass_scale = r.mass_scale;
    if (f64)
      k_pack_f64<<<grid1d(s.n), 256, 0, c->stream>>>(p, pc.rec.as<double4>(), pc.ext.as<double>());
    else
      k_pack_f32<<<grid1d(s.n), 256, 0, c->stream>>>(p, pc.rec.as<float4>(), pc.ext.as<float>());
    COUNT_LAUNCH(c);
    CUDA_TRY(c, cudaGetLastError());
  }
  pc.key = key;
  return BBKDE_OK;
}

// Query coordinates of `set` (QUERY, or REFERENCE for self-evaluation).
int ensure_queries(bbkde_ctx *c, int set, bool f64, const void **qx, const void **qy) {
  PointSet &s = c->sets[set];
  if (f64) {
    *qx = s.x.p;
    *qy = s.dim == 2 ? s.y.p : s.x.p;
    return BBKDE_OK;
  }
  QueryCache &qc = c->q32[set];
  if (!(qc.set == set && qc.coord_version == s.coord_version)) {
    const int64_t n = std::max<int64_t>(s.n, 1);
    TRY(ensure(c, qc.x, (size_t)n * sizeof(float)));
    TRY(ensure(c, qc.y, (size_t)n * sizeof(float)));
    if (s.n > 0) {
      k_to_f32<<<grid1d(s.n), 256, 0, c->stream>>>(s.x.as<double>(), qc.x.as<float>(), s.n);
      COUNT_LAUNCH(c);
      if (s.dim == 2) {
        k_to_f32<<<grid1d(s.n), 256, 0, c->stream>>>(s.y.as<double>(), qc.y.as<float>(), s.n);
        COUNT_LAUNCH(c);
      }
      CUDA_TRY(c, cudaGetLastError());
    }
    qc.set = set;
    qc.coord_version = s.coord_version;
  }
  *qx = qc.x.p;
  *qy = s.dim == 2 ? qc.y.p : qc.x.p;
  return BBKDE_OK;
}

// ---- launch planning ------------------------------------------------------

// Launch shapes of the FP32 pair-sum kernels. The autotuner times them on a
// slice of the actual problem and keeps the fastest per problem class.
struct Variant {
  int qpt;     // queries per thread
  int block;   // threads per block
  int minb;    // __launch_bounds__ minimum resident blocks per SM
  int poly;    // every poly-th reference's exponentials on the FP32 pipe (0: none)
};
constexpr Variant kVariants[] = {{8, 256, 2, 0},  {4, 256, 3, 0},  {8, 128, 4, 0},
                                 {4, 128, 6, 0},  {8, 256, 2, 8},  {8, 128, 4, 8},
                                 {8, 128, 4, 4},  {4, 128, 6, 8},  {4, 128, 6, 16},
                                 {4, 128, 6, 32}, {8, 256, 2, 16}};
constexpr int kNumVariants = 11;
constexpr int kDefaultVariant = 0;
constexpr int kTile = 256;
constexpr int kBlock64 = 128;
// Problems below this many pairs skip autotuning (launch-latency bound anyway).
constexpr double kAutotuneMinPairs = 2.0e10;

inline int queries_per_block(int variant, bool f64) {
  if (f64) return kBlock64;
  return kVariants[variant].qpt * kVariants[variant].block;
}

struct Plan {
  int64_t nseg = 1, seg_len = 0;
  unsigned gx = 1;
};

// Split the reference range into segments so that the grid fills the device
// with ~16 waves of blocks (load balance through the hardware block scheduler),
// but never below one staging tile of references per segment (small problems:
// 10,000 x 10,000 pairs would otherwise run on half the SMs).
Plan plan_launch(const bbkde_ctx *c, int64_t n_ref, int64_t q_count, int q_per_block,
                 int tile) {
  Plan p;
  int64_t qtiles = (q_count + q_per_block - 1) / q_per_block;
  p.gx = (unsigned)std::max<int64_t>(qtiles, 1);
  int64_t target = (int64_t)c->sm_count * 4 * 16;
  int64_t want = (target + qtiles - 1) / std::max<int64_t>(qtiles, 1);
  int64_t max_seg = std::max<int64_t>(1, (n_ref + tile - 1) / tile);
  p.nseg = std::min<int64_t>(std::max<int64_t>(want, 1), std::min<int64_t>(max_seg, 65535));
  p.seg_len = (n_ref + p.nseg - 1) / p.nseg;
  p.seg_len = (p.seg_len + tile - 1) / tile * tile;
  p.nseg = std::max<int64_t>(1, (n_ref + p.seg_len - 1) / p.seg_len);
  return p;
}

template <int OP, int D, int QPT, int BLOCK, int MINB, int POLY = 0>
void launch_shape(dim3 grid, cudaStream_t st, const SumArgs &a) {
  if constexpr (op_packed(OP))
    k_pair_sum_f32x2<OP, D, QPT, BLOCK, kTile, MINB, POLY><<<grid, BLOCK, 0, st>>>(a);
  else
    k_pair_sum_f32<OP, D, QPT, BLOCK, kTile, MINB><<<grid, BLOCK, 0, st>>>(a);
}

template <int OP, int D>
void launch_f32(int variant, dim3 grid, cudaStream_t st, const SumArgs &a) {
  switch (variant) {
    case 0: launch_shape<OP, D, 8, 256, 2>(grid, st, a); break;
    case 1: launch_shape<OP, D, 4, 256, 3>(grid, st, a); break;
    case 2: launch_shape<OP, D, 8, 128, 4>(grid, st, a); break;
    case 3: launch_shape<OP, D, 4, 128, 6>(grid, st, a); break;
    case 4: launch_shape<OP, D, 8, 256, 2, 8>(grid, st, a); break;
    case 5: launch_shape<OP, D, 8, 128, 4, 8>(grid, st, a); break;
    case 6: launch_shape<OP, D, 8, 128, 4, 4>(grid, st, a); break;
    case 7: launch_shape<OP, D, 4, 128, 6, 8>(grid, st, a); break;
    case 8: launch_shape<OP, D, 4, 128, 6, 16>(grid, st, a); break;
    case 9: launch_shape<OP, D, 4, 128, 6, 32>(grid, st, a); break;
    default: launch_shape<OP, D, 8, 256, 2, 16>(grid, st, a); break;
  }
}
template <int OP, int D>
void launch_f64(dim3 grid, cudaStream_t st, const SumArgs &a) {
  k_pair_sum_f64<OP, D, kBlock64><<<grid, kBlock64, 0, st>>>(a);
}

template <int D>
void dispatch_op(int op, bool f64, int variant, dim3 grid, cudaStream_t st, const SumArgs &a) {
  switch (op) {
#define CASE_(OPV)                                         \
  case OPV:                                                \
    if (f64) launch_f64<OPV, D>(grid, st, a);              \
    else launch_f32<OPV, D>(variant, grid, st, a);         \
    break;
    CASE_(OP_GAUSS_ISO)
    CASE_(OP_GAUSS_PROD)
    CASE_(OP_EPAN_ISO)
    CASE_(OP_EPAN_PROD)
    CASE_(OP_EPAN_CONV)
#undef CASE_
  }
}

inline int ilog2(int64_t v) {
  int r = 0;
  while (v > 1) { v >>= 1; ++r; }
  return r;
}

// Fill SumArgs and launch one pair-sum kernel over [r_i, r_j] x [q_i, q_j].
int launch_pair_sum(bbkde_ctx *c, const Resolved &r, bool f64, int variant, const void *qx,
                    const void *qy, int64_t r_i, int64_t r_j, int64_t q_i, int64_t q_j,
                    bool exclude_self, double scale, double *out, int64_t *nseg_out) {
  const int64_t n_ref = r_j - r_i + 1;
  const int64_t q_count = q_j - q_i + 1;
  Plan p = plan_launch(c, n_ref, q_count, queries_per_block(variant, f64),
                       f64 ? kBlock64 : kTile);
  PackCache &pc = f64 ? c->pack64 : c->pack32;
  SumArgs a;
  a.refs = pc.rec.p;
  a.extra = pc.ext.p;
  a.qx = qx;
  a.qy = qy;
  a.r_begin = r_i;
  a.r_end = r_j + 1;
  a.seg_len = p.seg_len;
  a.q_begin = q_i;
  a.q_count = q_count;
  a.exclude_self = exclude_self ? 1 : 0;
  a.scale = scale;
  a.out = out;
  a.status = c->status.as<int>();
  if (nseg_out) *nseg_out = p.nseg;
  if (!out) return BBKDE_OK;   // planning only
  dim3 grid(p.gx, (unsigned)p.nseg);
  if (r.dim == 2) dispatch_op<2>(r.op, f64, variant, grid, c->stream, a);
  else dispatch_op<1>(r.op, f64, variant, grid, c->stream, a);
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  return BBKDE_OK;
}

// Pick the FP32 launch shape: forced, cached, or timed on a slice of the problem
// (up to 131072 queries x 262144 references, every variant twice, fastest kept).
int choose_variant(bbkde_ctx *c, const Resolved &r, const void *qx, const void *qy,
                   int64_t r_i, int64_t r_j, int64_t q_i, int64_t q_j, bool exclude_self,
                   int *variant) {
  if (c->forced_variant >= 0) { *variant = c->forced_variant; return BBKDE_OK; }
  const double pairs = (double)(r_j - r_i + 1) * (double)(q_j - q_i + 1);
  if (pairs < kAutotuneMinPairs) { *variant = kDefaultVariant; return BBKDE_OK; }
  auto key = std::make_tuple(r.op, r.dim, exclude_self ? 1 : 0, ilog2(r_j - r_i + 1),
                             ilog2(q_j - q_i + 1));
  auto it = c->tuned.find(key);
  if (it != c->tuned.end()) { *variant = it->second; return BBKDE_OK; }
  const int64_t sq_j = std::min<int64_t>(q_j, q_i + 131072 - 1);
  const int64_t sr_j = std::min<int64_t>(r_j, r_i + 262144 - 1);
  int64_t need = 0;
  for (int v = 0; v < kNumVariants; ++v) {
    int64_t nseg = 0;
    TRY(launch_pair_sum(c, r, false, v, qx, qy, r_i, sr_j, q_i, sq_j, exclude_self, 1.0,
                        nullptr, &nseg));
    need = std::max<int64_t>(need, nseg * (sq_j - q_i + 1));
  }
  TRY(ensure(c, c->partial, (size_t)need * sizeof(double)));
  float best_ms = 0.f;
  int best = kDefaultVariant;
  for (int v = 0; v < kNumVariants; ++v) {
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
      TRY(launch_pair_sum(c, r, false, v, qx, qy, r_i, sr_j, q_i, sq_j, exclude_self, 1.0,
                          c->partial.as<double>(), nullptr));
      CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
      CUDA_TRY(c, cudaEventSynchronize(c->ev1));
      CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    }
    if (v == 0 || ms < best_ms) { best_ms = ms; best = v; }
  }
  c->tuned[key] = best;
  *variant = best;
  return BBKDE_OK;
}

// One pair-sum over refs [r_i, r_j] x queries [q_i, q_j] of `qset`; writes
// scale * sum into out_dev[0 .. q_count). With epi != EPI_NONE also reduces
// sum_q w[q] * g(out[q]) into c->scalars[0] (FP64, fixed order).
int pair_sum(bbkde_ctx *c, const Resolved &r, int precision, int qset, int64_t r_i,
             int64_t r_j, int64_t q_i, int64_t q_j, double scale, bool exclude_self,
             double *out_dev, int epi, const double *w_dev) {
  const bool f64 = precision == BBKDE_FP64;
  TRY(ensure_pack(c, r, f64));
  const void *qx = nullptr, *qy = nullptr;
  TRY(ensure_queries(c, qset, f64, &qx, &qy));
  const int64_t n_ref = r_j - r_i + 1;
  const int64_t q_count = q_j - q_i + 1;
  int variant = 0;
  if (!f64) TRY(choose_variant(c, r, qx, qy, r_i, r_j, q_i, q_j, exclude_self, &variant));
  int64_t nseg = 1;
  TRY(launch_pair_sum(c, r, f64, variant, qx, qy, r_i, r_j, q_i, q_j, exclude_self, 1.0,
                      nullptr, &nseg));
  double *partial = out_dev;
  const bool combine = nseg > 1 || epi != EPI_NONE;
  if (combine) {
    TRY(ensure(c, c->partial, (size_t)nseg * q_count * sizeof(double)));
    partial = c->partial.as<double>();
  }
  CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
  TRY(launch_pair_sum(c, r, f64, variant, qx, qy, r_i, r_j, q_i, q_j, exclude_self,
                      combine ? 1.0 : scale, partial, nullptr));
  CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
  int64_t launches = 1;
  if (combine) {
    const unsigned nb = grid1d(q_count, kRedBlock);
    if (epi != EPI_NONE) TRY(ensure(c, c->block_sums, (size_t)nb * sizeof(double)));
    k_combine<<<nb, kRedBlock, 0, c->stream>>>(partial, (int)nseg, q_count, scale, out_dev,
                                               epi, w_dev, c->block_sums.as<double>());
    COUNT_LAUNCH(c);
    CUDA_TRY(c, cudaGetLastError());
    ++launches;
    if (epi != EPI_NONE) {
      k_sum_blocks<<<1, kRedBlock, 0, c->stream>>>(c->block_sums.as<double>(), nb,
                                                   c->scalars.as<double>());
      COUNT_LAUNCH(c);
      CUDA_TRY(c, cudaGetLastError());
      ++launches;
    }
  }
  CUDA_TRY(c, cudaEventRecord(c->ev2, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  c->last_pairs = (double)n_ref * (double)q_count;
  c->last_launches = launches;
  c->last_variant = f64 ? -1 : variant;
  return BBKDE_OK;
}

int check_ranges(bbkde_ctx *c, int64_t r_i, int64_t r_j, int64_t q_i, int64_t q_j) {
  const int64_t nr = c->sets[BBKDE_REFERENCE].n, nq = c->sets[BBKDE_QUERY].n;
  // CudaDirectKde.h:181-190 (unsigned size_t there; negative indices here are
  // out of range as well).
  if (r_j >= nr || q_j >= nq || r_i < 0 || q_i < 0 || r_j < 0 || q_j < 0)
    return fail(c, BBKDE_OUT_OF_RANGE,
                "CudaDirectKde<>: unnormalized_eval(): j_r and j_q should be at most "
                "the number of reference and query points. ");
  if (r_i > r_j || q_i > q_j)
    return fail(c, BBKDE_INVALID_ARGUMENT,
                "CudaDirectKde<>: unnormalized_eval(): must have i_r <= j_r and i_q <= j_q. ");
  return BBKDE_OK;
}

int eval_common(bbkde_ctx *c, const bbkde_kernel_desc *k, int64_t r_i, int64_t r_j,
                int64_t q_i, int64_t q_j, int normalized, int precision, double *out,
                bool out_is_device) {
  TRY(check_ctx(c));
  if (!out) return fail(c, BBKDE_INVALID_ARGUMENT, "output pointer is NULL");
  if (precision != BBKDE_FP32C && precision != BBKDE_FP64)
    return fail(c, BBKDE_INVALID_ARGUMENT, "unknown precision");
  Resolved r;
  TRY(resolve(c, k, r));
  TRY(check_ranges(c, r_i, r_j, q_i, q_j));
  if (c->sets[BBKDE_REFERENCE].dim != r.dim || c->sets[BBKDE_QUERY].dim != r.dim)
    return fail(c, BBKDE_INVALID_ARGUMENT, "point dimension does not match the kernel");
  const int64_t q_count = q_j - q_i + 1;
  double *dst = out;
  if (!out_is_device) {
    TRY(ensure(c, c->out_dev, (size_t)q_count * sizeof(double)));
    dst = c->out_dev.as<double>();
  }
  TRY(pair_sum(c, r, precision, BBKDE_QUERY, r_i, r_j, q_i, q_j,
               normalized ? r.norm : 1.0, false, dst, EPI_NONE, nullptr));
  if (!out_is_device) {
    CUDA_TRY(c, cudaMemcpyAsync(out, dst, (size_t)q_count * sizeof(double),
                                cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  return BBKDE_OK;
}

int download(bbkde_ctx *c, double *host, const DevBuf &src, int64_t n) {
  if (!host || n <= 0) return BBKDE_OK;
  CUDA_TRY(c, cudaMemcpyAsync(host, src.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  return BBKDE_OK;
}

int self_checks(bbkde_ctx *c, const bbkde_kernel_desc *k, int precision, Resolved &r) {
  TRY(check_ctx(c));
  if (precision != BBKDE_FP32C && precision != BBKDE_FP64)
    return fail(c, BBKDE_INVALID_ARGUMENT, "unknown precision");
  TRY(resolve(c, k, r));
  const PointSet &s = c->sets[BBKDE_REFERENCE];
  if (s.dim != r.dim && s.n > 0)
    return fail(c, BBKDE_INVALID_ARGUMENT, "point dimension does not match the kernel");
  return BBKDE_OK;
}

int conv_kind_of(int kind, int dim) {
  if (dim == 1 && kind == BBKDE_GAUSSIAN) return BBKDE_GAUSSIAN_CONV_1D;
  if (dim == 1 && kind == BBKDE_EPANECHNIKOV) return BBKDE_EPANECHNIKOV_CONV_1D;
  if (kind == BBKDE_GAUSSIAN_PRODUCT_2D) return BBKDE_GAUSSIAN_PRODUCT_CONV_2D;
  if (kind == BBKDE_EPANECHNIKOV_PRODUCT_2D) return BBKDE_EPANECHNIKOV_PRODUCT_CONV_2D;
  return -1;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int bbkde_abi_version(void) { return BBKDE_ABI_VERSION; }

const char *bbkde_status_string(int s) {
  switch (s) {
    case BBKDE_OK: return "ok";
    case BBKDE_OUT_OF_RANGE: return "out of range";
    case BBKDE_INVALID_ARGUMENT: return "invalid argument";
    case BBKDE_CUDA_ERROR: return "CUDA error";
    case BBKDE_TIMEOUT: return "timeout";
    case BBKDE_UNSUPPORTED: return "unsupported";
    case BBKDE_NO_DEVICE: return "no CUDA device";
    case BBKDE_ALLOC_FAILED: return "device allocation failed";
  }
  return "unknown status";
}

int bbkde_ctx_create(int device, bbkde_ctx **out) {
  if (!out) return BBKDE_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return BBKDE_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return BBKDE_INVALID_ARGUMENT;
  bbkde_ctx *c = new (std::nothrow) bbkde_ctx();
  if (!c) return BBKDE_ALLOC_FAILED;
  c->device = device;
  int rc = BBKDE_OK;
  do {
    if (cudaSetDevice(device) != cudaSuccess) { rc = BBKDE_CUDA_ERROR; break; }
    if (cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device) !=
            cudaSuccess ||
        c->sm_count < 1) {
      rc = BBKDE_CUDA_ERROR;
      break;
    }
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
      rc = BBKDE_CUDA_ERROR;
      break;
    }
    c->stream = c->own_stream;
    if (cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->ev2) != cudaSuccess || cudaEventCreate(&c->ev3) != cudaSuccess) {
      rc = BBKDE_CUDA_ERROR;
      break;
    }
    if ((rc = ensure(c, c->scalars, 64 * sizeof(double))) != BBKDE_OK) break;
    if ((rc = ensure(c, c->status, 64)) != BBKDE_OK) break;
    if (cudaMemset(c->status.p, 0, 64) != cudaSuccess) { rc = BBKDE_CUDA_ERROR; break; }
  } while (0);
  if (rc != BBKDE_OK) {
    cudaGetLastError();
    bbkde_ctx_destroy(c);
    return rc;
  }
  *out = c;
  return BBKDE_OK;
}

int bbkde_ctx_destroy(bbkde_ctx *c) {
  if (!c) return BBKDE_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto &s : c->sets) {
    release(s.x); release(s.y); release(s.mass); release(s.abw); release(s.weight);
  }
  release(c->pack32.rec); release(c->pack32.ext);
  release(c->pack64.rec); release(c->pack64.ext);
  for (auto &q : c->q32) { release(q.x); release(q.y); }
  release(c->partial); release(c->out_dev); release(c->block_sums);
  release(c->scalars); release(c->staging); release(c->status);
  for (DevBuf *b : {&c->cv_x, &c->cv_y, &c->cv_w, &c->cv_cells, &c->cv_sets, &c->cv_items,
                    &c->cv_counter, &c->cv_h, &c->cv_lut, &c->cv_part, &c->cv_hist,
                    &c->cv_out, &c->cv_parts})
    release(*b);
  for (DevBuf *b : {&c->cull.rec, &c->cull.ext, &c->cull.tiles, &c->cull.groups, &c->ms_keys,
                    &c->ms_keys2, &c->ms_perm, &c->ms_perm2, &c->ms_box, &c->ms_tmp, &c->cq_x,
                    &c->cq_y, &c->cq_out, &c->cb_bound, &c->cb_smin, &c->cb_tiles, &c->cb_stats,
                    &c->cb_key, &c->cb_key2, &c->cb_sched,
                    &c->gr_pred, &c->gr_order, &c->gr_tmin, &c->gr_tmax, &c->gr_bad,
                    &c->gr_terr, &c->gr_flag, &c->gr_flag_ord, &c->gr_list, &c->gr_nsel,
                    &c->gr_counts, &c->gr_gmax, &c->gr_lat_order, &c->gr_lat_exact,
                    &c->gr_lat_net, &c->gr_q_order, &c->gr_q_exact, &c->gr_q_net, &c->gr_resid,
                    &c->gr_cand_ord, &c->gr_cand_xy, &c->gr_cand_net, &c->gr_out,
                    &c->gr_part, &c->gr_rl_idx, &c->gr_rl_xy, &c->gr_rl_net})
    release(*b);
  if (c->cv_graph) cudaGraphExecDestroy(c->cv_graph);
  if (c->ev3) cudaEventDestroy(c->ev3);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev2) cudaEventDestroy(c->ev2);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return BBKDE_OK;
}

const char *bbkde_ctx_last_error(const bbkde_ctx *c) {
  return c ? c->err.c_str() : "null context";
}

int bbkde_ctx_set_stream(bbkde_ctx *c, void *stream) {
  TRY(check_ctx(c));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
  return BBKDE_OK;
}

int bbkde_upload(bbkde_ctx *c, int role, int dim, int64_t n, const double *coords,
                 const double *mass, const double *abw, const double *weight) {
  TRY(check_ctx(c));
  if (role != BBKDE_REFERENCE && role != BBKDE_QUERY)
    return fail(c, BBKDE_INVALID_ARGUMENT, "role must be REFERENCE or QUERY");
  if (dim != 1 && dim != 2) return fail(c, BBKDE_INVALID_ARGUMENT, "dim must be 1 or 2");
  if (n < 0) return fail(c, BBKDE_INVALID_ARGUMENT, "negative point count");
  if (n > 0 && !coords) return fail(c, BBKDE_INVALID_ARGUMENT, "coords is NULL");
  PointSet &s = c->sets[role];
  const size_t nb = (size_t)std::max<int64_t>(n, 1) * sizeof(double);
  TRY(ensure(c, s.x, nb));
  TRY(ensure(c, s.y, nb));
  TRY(ensure(c, s.mass, nb));
  TRY(ensure(c, s.abw, nb));
  TRY(ensure(c, s.weight, nb));
  TRY(ensure(c, c->staging, nb * dim));
  if (n > 0) {
    CUDA_TRY(c, cudaMemcpyAsync(c->staging.p, coords, (size_t)n * dim * sizeof(double),
                                cudaMemcpyHostToDevice, c->stream));
    k_deinterleave<<<grid1d(n), 256, 0, c->stream>>>(c->staging.as<double>(), dim, n,
                                                     s.x.as<double>(), s.y.as<double>());
    COUNT_LAUNCH(c);
    CUDA_TRY(c, cudaGetLastError());
    if (mass)
      CUDA_TRY(c, cudaMemcpyAsync(s.mass.p, mass, nb, cudaMemcpyHostToDevice, c->stream));
    else
      k_fill<<<grid1d(n), 256, 0, c->stream>>>(s.mass.as<double>(), 1.0, n), COUNT_LAUNCH(c);
    if (abw)
      CUDA_TRY(c, cudaMemcpyAsync(s.abw.p, abw, nb, cudaMemcpyHostToDevice, c->stream));
    else
      k_fill<<<grid1d(n), 256, 0, c->stream>>>(s.abw.as<double>(), 1.0, n), COUNT_LAUNCH(c);
    if (weight)
      CUDA_TRY(c, cudaMemcpyAsync(s.weight.p, weight, nb, cudaMemcpyHostToDevice, c->stream));
    else
      CUDA_TRY(c, cudaMemcpyAsync(s.weight.p, s.mass.p, nb, cudaMemcpyDeviceToDevice,
                                  c->stream));
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  s.dim = dim;
  s.n = n;
  ++s.coord_version;
  ++s.attr_version;
  return BBKDE_OK;
}

int64_t bbkde_size(const bbkde_ctx *c, int role) {
  if (!c || (role != BBKDE_REFERENCE && role != BBKDE_QUERY)) return -1;
  return c->sets[role].n;
}

int bbkde_download_attributes(bbkde_ctx *c, double *mass, double *abw) {
  TRY(check_ctx(c));
  const PointSet &s = c->sets[BBKDE_REFERENCE];
  TRY(download(c, mass, s.mass, s.n));
  TRY(download(c, abw, s.abw, s.n));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return BBKDE_OK;
}

int bbkde_eval_range(bbkde_ctx *c, const bbkde_kernel_desc *k, int64_t r_i, int64_t r_j,
                     int64_t q_i, int64_t q_j, int normalized, int precision, double *out,
                     int64_t block_size) {
  (void)block_size;
  return eval_common(c, k, r_i, r_j, q_i, q_j, normalized, precision, out, false);
}

int bbkde_eval_range_device(bbkde_ctx *c, const bbkde_kernel_desc *k, int64_t r_i,
                            int64_t r_j, int64_t q_i, int64_t q_j, int normalized,
                            int precision, double *out_device, int64_t block_size) {
  (void)block_size;
  return eval_common(c, k, r_i, r_j, q_i, q_j, normalized, precision, out_device, true);
}

int bbkde_unadapt_density(bbkde_ctx *c) {
  TRY(check_ctx(c));
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (s.n > 0) {
    k_unadapt<<<grid1d(s.n), 256, 0, c->stream>>>(s.weight.as<double>(), s.n,
                                                  s.abw.as<double>(), s.mass.as<double>());
    COUNT_LAUNCH(c);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  }
  ++s.attr_version;
  return BBKDE_OK;
}

int bbkde_adapt_density(bbkde_ctx *c, const bbkde_kernel_desc *k, double alpha, int precision,
                        double *abw_out, double *mass_out, double *pilot_out, double *g_out) {
  Resolved r;
  TRY(self_checks(c, k, precision, r));
  // KernelDensityImpl.h:301-303
  if (!(alpha >= 0 && alpha <= 1))
    return fail(c, BBKDE_INVALID_ARGUMENT, "adapt_density: alpha must be between [0, 1]. ");
  TRY(bbkde_unadapt_density(c));  // :307
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (alpha == 0 || s.n == 0) {    // :311
    if (g_out) *g_out = NAN;
    TRY(download(c, abw_out, s.abw, s.n));
    TRY(download(c, mass_out, s.mass, s.n));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BBKDE_OK;
  }
  // Pilot: all-pairs self-evaluation with the self term (:319-325).
  TRY(ensure(c, c->out_dev, (size_t)s.n * sizeof(double)));
  double *pilot = c->out_dev.as<double>();
  TRY(pair_sum(c, r, precision, BBKDE_REFERENCE, 0, s.n - 1, 0, s.n - 1, r.norm, false, pilot,
               EPI_W_LOG, s.weight.as<double>()));
  const double ms = c->last_ms, pairs = c->last_pairs;
  const int64_t launches = c->last_launches;
  // g, local bandwidths, masses (:330-353).
  k_pilot_finalize<<<grid1d(s.n), 256, 0, c->stream>>>(
      pilot, s.weight.as<double>(), c->scalars.as<double>(), alpha, r.dim, s.n,
      s.abw.as<double>(), s.mass.as<double>(), c->scalars.as<double>() + 1);
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  ++s.attr_version;
  TRY(download(c, pilot_out, c->out_dev, s.n));
  TRY(download(c, abw_out, s.abw, s.n));
  TRY(download(c, mass_out, s.mass, s.n));
  double g = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&g, c->scalars.as<double>() + 1, sizeof(double),
                              cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (g_out) *g_out = g;
  c->last_ms = ms;
  c->last_pairs = pairs;
  c->last_launches = launches + 1;
  return BBKDE_OK;
}

int bbkde_likelihood_cv(bbkde_ctx *c, const bbkde_kernel_desc *k, int precision,
                        double *cv_out) {
  Resolved r;
  TRY(self_checks(c, k, precision, r));
  if (!cv_out) return fail(c, BBKDE_INVALID_ARGUMENT, "cv_out is NULL");
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (s.n == 0) { *cv_out = 0.0; return BBKDE_OK; }
  TRY(ensure(c, c->out_dev, (size_t)s.n * sizeof(double)));
  TRY(pair_sum(c, r, precision, BBKDE_REFERENCE, 0, s.n - 1, 0, s.n - 1, r.norm, true,
               c->out_dev.as<double>(), EPI_W_LOG, s.weight.as<double>()));
  CUDA_TRY(c, cudaMemcpy(cv_out, c->scalars.p, sizeof(double), cudaMemcpyDeviceToHost));
  return BBKDE_OK;
}

int bbkde_lsq_conv_cv(bbkde_ctx *c, const bbkde_kernel_desc *k, int precision, double *cv_out) {
  Resolved r;
  TRY(self_checks(c, k, precision, r));
  if (!cv_out) return fail(c, BBKDE_INVALID_ARGUMENT, "cv_out is NULL");
  const int ck = conv_kind_of(k->kind, k->dim);
  if (ck < 0)
    return fail(c, BBKDE_UNSUPPORTED, "no convolution kernel is associated with this kernel");
  bbkde_kernel_desc kc = *k;
  kc.kind = ck;
  Resolved rc;
  TRY(resolve(c, &kc, rc));
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (s.n == 0) { *cv_out = 0.0; return BBKDE_OK; }
  TRY(ensure(c, c->out_dev, (size_t)s.n * sizeof(double)));
  double llo = 0, sq = 0;
  // Leave-one-out term (:162-181).
  TRY(pair_sum(c, r, precision, BBKDE_REFERENCE, 0, s.n - 1, 0, s.n - 1, r.norm, true,
               c->out_dev.as<double>(), EPI_W_VALUE, s.weight.as<double>()));
  CUDA_TRY(c, cudaMemcpy(&llo, c->scalars.p, sizeof(double), cudaMemcpyDeviceToHost));
  const double ms = c->last_ms;
  // Square-integral term with the convolution kernel, all pairs (:187-205).
  TRY(pair_sum(c, rc, precision, BBKDE_REFERENCE, 0, s.n - 1, 0, s.n - 1, rc.norm, false,
               c->out_dev.as<double>(), EPI_W_VALUE, s.weight.as<double>()));
  CUDA_TRY(c, cudaMemcpy(&sq, c->scalars.p, sizeof(double), cudaMemcpyDeviceToHost));
  c->last_ms += ms;
  c->last_pairs *= 2;
  *cv_out = sq - 2 * llo;  // :207
  return BBKDE_OK;
}

int bbkde_last_launch_stats(const bbkde_ctx *c, double *kernel_ms, double *pairs,
                            int64_t *launches) {
  if (!c) return BBKDE_INVALID_ARGUMENT;
  if (kernel_ms) *kernel_ms = c->last_ms;
  if (pairs) *pairs = c->last_pairs;
  if (launches) *launches = c->last_launches;
  return BBKDE_OK;
}

int64_t bbkde_launch_count(const bbkde_ctx *c) { return c ? c->launch_total : -1; }

int bbkde_ctx_set_launch_variant(bbkde_ctx *c, int variant) {
  if (!c) return BBKDE_INVALID_ARGUMENT;
  if (variant < -1 || variant >= kNumVariants)
    return fail(c, BBKDE_INVALID_ARGUMENT, "launch variant out of range");
  c->forced_variant = variant;
  return BBKDE_OK;
}

int bbkde_launch_variants(const bbkde_ctx *c, int *n_variants, int *last_variant) {
  if (!c) return BBKDE_INVALID_ARGUMENT;
  if (n_variants) *n_variants = kNumVariants;
  if (last_variant) *last_variant = c->last_variant;
  return BBKDE_OK;
}

int bbkde_device_info(const bbkde_ctx *c, int *sm_count, int *device) {
  if (!c) return BBKDE_INVALID_ARGUMENT;
  if (sm_count) *sm_count = c->sm_count;
  if (device) *device = c->device;
  return BBKDE_OK;
}

}  // extern "C"

// ===========================================================================
// Batched cross-validation (bbkde_cv_batch)
// ===========================================================================
namespace {

constexpr int kCvBlock = 1024;

// Work-item plans of the batched CV launch: likelihood items of `chunk` queries
// of one set, convolution items of at most `qblock` (<= kCvQBlock) queries of one
// grid cell. Smaller items balance the 148 persistent blocks better at the end of
// the launch; larger ones pay the per-item histogram set-up and flush less often.
struct CvPlan {
  int chunk, qblock;
};
constexpr CvPlan kCvPlans[] = {{4096, 256}, {1024, 256}, {2048, 128}};
constexpr int kCvNumPlans = 3;

size_t cv_smem_bytes() {
  return sizeof(double) * (4 * kCvHist + 6 * kCvMaxH + 3 * kCvQBlock) +
         sizeof(int64_t) * (2 * kCvMaxRanges + 1) + 4 * sizeof(int) + 2 * kCvLut;
}

// Lower-bound table for cv_cell: bin i holds #{h[a] <= the smallest double whose
// key (bits >> shift) is base + i}. The shift keeps as many mantissa bits as fit
// kCvLut bins over [h_min / 4, h_max] (64 bins per octave for the usual grids).
void cv_lut(const double *h, int n, int shift, long long &base, unsigned char *lut) {
  auto key = [&](double v) {
    long long b;
    std::memcpy(&b, &v, sizeof(b));
    return b >> shift;
  };
  base = key(h[0] / 4.0);
  for (int i = 0; i < kCvLut; ++i) {
    long long bits = (base + i) << shift;
    double v;
    std::memcpy(&v, &bits, sizeof(v));
    int cnt = 0;
    while (cnt < n && h[cnt] <= v) ++cnt;
    lut[i] = (unsigned char)cnt;
  }
}

int cv_lut_shift(const double *hx, int nx, const double *hy, int ny) {
  const double lo = std::min(hx[0], hy[0]) / 4.0;
  const double hi = std::max(hx[nx - 1], hy[ny - 1]) * 1.01;
  const double octaves = std::log2(hi / lo) + 2.0;
  int mbits = 8;
  while (mbits > 0 && octaves * (1 << mbits) > kCvLut) --mbits;
  return 52 - mbits;
}

int cv_check_grid(bbkde_ctx *c, int n, const double *h, const char *name) {
  if (n < 1 || n > kCvMaxH || !h)
    return fail(c, BBKDE_INVALID_ARGUMENT,
                std::string(name) + ": between 1 and 64 bandwidths are supported");
  for (int i = 0; i < n; ++i) {
    if (!(h[i] > 0) || !std::isfinite(h[i]) || (i > 0 && !(h[i] > h[i - 1])))
      return fail(c, BBKDE_INVALID_ARGUMENT,
                  std::string(name) + ": bandwidths must be positive and strictly increasing");
  }
  return BBKDE_OK;
}

// Gaussian product kernel: exact per-bandwidth loop over the pair sum.
int cv_batch_loop(bbkde_ctx *c, int kind, int n_sets, const bbkde_dataset *sets, int n_hx,
                  const double *hx, int n_hy, const double *hy, int precision, double *lik,
                  double *lsq) {
  double ms = 0, pairs = 0;
  for (int sidx = 0; sidx < n_sets; ++sidx) {
    const bbkde_dataset &d = sets[sidx];
    std::vector<double> w(d.n);
    double tot = 0;
    for (int64_t i = 0; i < d.n; ++i) tot += d.weights ? d.weights[i] : 1.0;
    for (int64_t i = 0; i < d.n; ++i) w[i] = (d.weights ? d.weights[i] : 1.0) / tot;
    TRY(bbkde_upload(c, BBKDE_REFERENCE, 2, d.n, d.coords, w.data(), nullptr, w.data()));
    for (int a = 0; a < n_hx; ++a)
      for (int b = 0; b < n_hy; ++b) {
        bbkde_kernel_desc k = {kind, 2, {hx[a], hy[b]}, 0, 0};
        const int64_t o = ((int64_t)sidx * n_hx + a) * n_hy + b;
        TRY(bbkde_likelihood_cv(c, &k, precision, lik + o));
        ms += c->last_ms;
        TRY(bbkde_lsq_conv_cv(c, &k, precision, lsq + o));
        ms += c->last_ms;
        pairs += 3.0 * (double)d.n * (double)d.n;
      }
  }
  c->last_ms = ms;
  c->last_pairs = pairs;
  return BBKDE_OK;
}

}  // namespace

extern "C" int bbkde_cv_batch(bbkde_ctx *c, int kind, int n_sets, const bbkde_dataset *sets,
                              int n_hx, const double *hx, int n_hy, const double *hy,
                              int precision, double *lik_out, double *lsq_out) {
  TRY(check_ctx(c));
  if (n_sets < 0 || (n_sets > 0 && !sets) || !lik_out || !lsq_out)
    return fail(c, BBKDE_INVALID_ARGUMENT, "cv_batch: bad dataset or output pointers");
  if (precision != BBKDE_FP32C && precision != BBKDE_FP64)
    return fail(c, BBKDE_INVALID_ARGUMENT, "unknown precision");
  TRY(cv_check_grid(c, n_hx, hx, "hx"));
  TRY(cv_check_grid(c, n_hy, hy, "hy"));
  for (int sidx = 0; sidx < n_sets; ++sidx) {
    if (sets[sidx].n < 2 || !sets[sidx].coords)
      return fail(c, BBKDE_INVALID_ARGUMENT, "cv_batch: every dataset needs at least 2 points");
  }
  if (kind == BBKDE_GAUSSIAN_PRODUCT_2D)
    return cv_batch_loop(c, kind, n_sets, sets, n_hx, hx, n_hy, hy, precision, lik_out,
                         lsq_out);
  if (kind != BBKDE_EPANECHNIKOV_PRODUCT_2D)
    return fail(c, BBKDE_UNSUPPORTED,
                "cv_batch: supported kernels are the 2-D Epanechnikov and Gaussian products");
  if (n_sets == 0) return BBKDE_OK;

  // ---- host: normalise weights, bin points on a grid, sort by cell --------
  const double hmax = std::max(hx[n_hx - 1], hy[n_hy - 1]);
  std::vector<CvSet> hs(n_sets);
  std::vector<double> X, Y, Wt;
  std::vector<int64_t> cells;
  int64_t total = 0;
  for (int sidx = 0; sidx < n_sets; ++sidx) total += sets[sidx].n;
  X.reserve(total); Y.reserve(total); Wt.reserve(total);
  double sum_pairs = 0;
  for (int sidx = 0; sidx < n_sets; ++sidx) {
    const bbkde_dataset &d = sets[sidx];
    const int64_t n = d.n;
    double xmin = d.coords[0], xmax = xmin, ymin = d.coords[1], ymax = ymin, wt = 0;
    for (int64_t i = 0; i < n; ++i) {
      const double x = d.coords[2 * i], y = d.coords[2 * i + 1];
      if (!std::isfinite(x) || !std::isfinite(y))
        return fail(c, BBKDE_INVALID_ARGUMENT, "cv_batch: non-finite coordinate");
      xmin = std::min(xmin, x); xmax = std::max(xmax, x);
      ymin = std::min(ymin, y); ymax = std::max(ymax, y);
      wt += d.weights ? d.weights[i] : 1.0;
    }
    if (!(wt > 0)) return fail(c, BBKDE_INVALID_ARGUMENT, "cv_batch: weights must sum > 0");
    // Cells of a quarter of the largest bandwidth, at most 4096 per axis.
    const double spread = std::max(xmax - xmin, ymax - ymin);
    const double cell = std::max(hmax / 4.0, spread / 4095.0);
    CvSet &s = hs[sidx];
    s.begin = (int64_t)X.size();
    s.n = n;
    s.cell_begin = (int64_t)cells.size();
    s.x0 = xmin;
    s.y0 = ymin;
    s.inv_cell = 1.0 / cell;
    s.gx = (int)std::floor((xmax - xmin) * s.inv_cell) + 1;
    s.gy = (int)std::floor((ymax - ymin) * s.inv_cell) + 1;
    const int64_t ncell = (int64_t)s.gx * s.gy;
    // Sort key: the cell, then the Morton order of the position inside the cell
    // (16 bits per axis), so that consecutive points of a cell are neighbours.
    auto spread16 = [](uint32_t v) {
      v &= 0xffffu;
      v = (v | (v << 8)) & 0x00ff00ffu;
      v = (v | (v << 4)) & 0x0f0f0f0fu;
      v = (v | (v << 2)) & 0x33333333u;
      v = (v | (v << 1)) & 0x55555555u;
      return v;
    };
    std::vector<int64_t> cnt(ncell + 1, 0);
    std::vector<uint64_t> key(n);
    for (int64_t i = 0; i < n; ++i) {
      const double fx = (d.coords[2 * i] - xmin) * s.inv_cell;
      const double fy = (d.coords[2 * i + 1] - ymin) * s.inv_cell;
      const int cx = std::min(s.gx - 1, std::max(0, (int)std::floor(fx)));
      const int cy = std::min(s.gy - 1, std::max(0, (int)std::floor(fy)));
      const int64_t cell_id = (int64_t)cy * s.gx + cx;
      auto sub = [](double f) {
        return (uint32_t)std::min(65535.0, std::max(0.0, std::floor(f * 65536.0)));
      };
      key[i] = ((uint64_t)cell_id << 32) |
               (spread16(sub(fx - cx)) | (spread16(sub(fy - cy)) << 1));
      ++cnt[cell_id + 1];
    }
    for (int64_t k = 0; k < ncell; ++k) cnt[k + 1] += cnt[k];
    cells.insert(cells.end(), cnt.begin(), cnt.end());   // set-relative cell_start
    std::vector<int64_t> order(n);
    for (int64_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int64_t u, int64_t v) {
      return key[u] != key[v] ? key[u] < key[v] : u < v;
    });
    X.resize(s.begin + n); Y.resize(s.begin + n); Wt.resize(s.begin + n);
    double diag = 0;
    for (int64_t r = 0; r < n; ++r) {
      const int64_t i = order[r], at = s.begin + r;
      const double w = (d.weights ? d.weights[i] : 1.0) / wt;
      X[at] = d.coords[2 * i];
      Y[at] = d.coords[2 * i + 1];
      Wt[at] = w;
      diag += w * w;
    }
    s.diag_wm = diag;
    sum_pairs += (double)n * (double)n;
  }
  // Work-item plan: forced, or tuned per problem class on the real calls -- the
  // first calls of a class each run an untried plan (every call returns complete
  // results whatever its plan; the likelihood sums' FP64 grouping follows the
  // plan), then the fastest measured plan is kept.
  const std::tuple<int, int, int, int, int> tkey{
      n_sets, (int)std::floor(std::log2((double)total)), n_hx, n_hy,
      (int)std::floor(std::log2(std::max(1.0, sum_pairs)))};
  int plan_id = 0;
  std::vector<double> *trials = nullptr;
  if (c->cv_forced_plan >= 0) {
    plan_id = c->cv_forced_plan;
  } else {
    trials = &c->cv_tuned[tkey];
    if (trials->empty()) trials->assign(kCvNumPlans, -1.0);
    int untried = -1;
    for (int i = 0; i < kCvNumPlans && untried < 0; ++i)
      if ((*trials)[i] < 0) untried = i;
    if (untried >= 0) {
      plan_id = untried;
    } else {
      for (int i = 1; i < kCvNumPlans; ++i)
        if ((*trials)[i] < (*trials)[plan_id]) plan_id = i;
      trials = nullptr;   // tuned: nothing more to record
    }
  }
  const CvPlan plan = kCvPlans[plan_id];
  // Work items: likelihood items (set, chunk of queries) and convolution items
  // (set, grid cell, block of <= plan.qblock queries, x-power group), ordered by
  // estimated cost so the largest start first.
  std::vector<CvItem> items;
  std::vector<double> cost;
  std::vector<int> part_begin(n_sets), part_count(n_sets);
  int parts = 0;
  for (int sidx = 0; sidx < n_sets; ++sidx) {
    const CvSet &st = hs[sidx];
    part_begin[sidx] = parts;
    part_count[sidx] = (int)((st.n + plan.chunk - 1) / plan.chunk);
    for (int ch = 0; ch < part_count[sidx]; ++ch) {
      const int64_t q0 = (int64_t)ch * plan.chunk;
      const int64_t q1 = std::min<int64_t>(st.n, q0 + plan.chunk);
      items.push_back({sidx, 0, parts + ch, 0, 0, 0, q0, q1});
      cost.push_back((double)(q1 - q0) * st.n);
    }
    parts += part_count[sidx];
    const int64_t *cst = cells.data() + st.cell_begin;
    for (int cy = 0; cy < st.gy; ++cy)
      for (int cx = 0; cx < st.gx; ++cx) {
        const int64_t cb = cst[(int64_t)cy * st.gx + cx], ce = cst[(int64_t)cy * st.gx + cx + 1];
        for (int64_t q0 = cb; q0 < ce; q0 += plan.qblock) {
          const int64_t q1 = std::min<int64_t>(ce, q0 + plan.qblock);
          for (int g = 0; g < 4; ++g) {
            items.push_back({sidx, 1 + g, 0, cx, cy, 0, q0, q1});
            cost.push_back(0.5 * (double)(q1 - q0) * st.n);
          }
        }
      }
  }
  {
    std::vector<size_t> idx(items.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](size_t p, size_t q) { return cost[p] > cost[q]; });
    std::vector<CvItem> sorted(items.size());
    for (size_t i = 0; i < idx.size(); ++i) sorted[i] = items[idx[i]];
    items.swap(sorted);
  }
  std::vector<double> hbuf(2 * kCvMaxH, 0.0);
  std::copy(hx, hx + n_hx, hbuf.begin());
  std::copy(hy, hy + n_hy, hbuf.begin() + kCvMaxH);
  std::vector<unsigned char> luts(2 * kCvLut);
  const int lut_shift = cv_lut_shift(hx, n_hx, hy, n_hy);
  long long basex = 0, basey = 0;
  cv_lut(hx, n_hx, lut_shift, basex, luts.data());
  cv_lut(hy, n_hy, lut_shift, basey, luts.data() + kCvLut);

  // ---- device buffers -----------------------------------------------------
  const size_t nb = (size_t)total * sizeof(double);
  TRY(ensure(c, c->cv_x, nb));
  TRY(ensure(c, c->cv_y, nb));
  TRY(ensure(c, c->cv_w, nb));
  TRY(ensure(c, c->cv_cells, cells.size() * sizeof(int64_t)));
  TRY(ensure(c, c->cv_sets, hs.size() * sizeof(CvSet)));
  TRY(ensure(c, c->cv_items, items.size() * sizeof(CvItem)));
  TRY(ensure(c, c->cv_counter, 64));
  TRY(ensure(c, c->cv_h, hbuf.size() * sizeof(double)));
  TRY(ensure(c, c->cv_lut, luts.size()));
  TRY(ensure(c, c->cv_part, (size_t)parts * 2 * kCvCells * sizeof(double)));
  TRY(ensure(c, c->cv_hist, (size_t)n_sets * 16 * kCvCells * sizeof(double)));
  const size_t nout = (size_t)n_sets * n_hx * n_hy;
  TRY(ensure(c, c->cv_out, 2 * nout * sizeof(double)));
  TRY(ensure(c, c->cv_parts, 2 * n_sets * sizeof(int)));
  std::vector<int> pinfo(part_begin);
  pinfo.insert(pinfo.end(), part_count.begin(), part_count.end());
  auto up = [&](DevBuf &b, const void *src, size_t bytes) {
    return cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->stream);
  };
  CUDA_TRY(c, up(c->cv_x, X.data(), nb));
  CUDA_TRY(c, up(c->cv_y, Y.data(), nb));
  CUDA_TRY(c, up(c->cv_w, Wt.data(), nb));
  CUDA_TRY(c, up(c->cv_cells, cells.data(), cells.size() * sizeof(int64_t)));
  CUDA_TRY(c, up(c->cv_sets, hs.data(), hs.size() * sizeof(CvSet)));
  CUDA_TRY(c, up(c->cv_items, items.data(), items.size() * sizeof(CvItem)));
  CUDA_TRY(c, up(c->cv_h, hbuf.data(), hbuf.size() * sizeof(double)));
  CUDA_TRY(c, up(c->cv_lut, luts.data(), luts.size()));
  CUDA_TRY(c, up(c->cv_parts, pinfo.data(), pinfo.size() * sizeof(int)));

  CvArgs a;
  a.x = c->cv_x.as<double>();
  a.y = c->cv_y.as<double>();
  a.w = c->cv_w.as<double>();
  a.m = c->cv_w.as<double>();   // non-adaptive: mass = weight
  a.cell_start = c->cv_cells.as<int64_t>();
  a.sets = c->cv_sets.as<CvSet>();
  a.items = c->cv_items.as<CvItem>();
  a.n_items = (int)items.size();
  a.counter = c->cv_counter.as<int>();
  a.nhx = n_hx;
  a.nhy = n_hy;
  a.hx = c->cv_h.as<double>();
  a.hy = c->cv_h.as<double>() + kCvMaxH;
  a.lutx = c->cv_lut.as<unsigned char>();
  a.luty = c->cv_lut.as<unsigned char>() + kCvLut;
  a.lut_basex = basex;
  a.lut_basey = basey;
  a.lut_shift = lut_shift;
  a.r_epan = 4;
  a.r_conv = 8;
  a.epan_part = c->cv_part.as<double>();
  a.conv_hist = c->cv_hist.as<double>();
  a.pairs = reinterpret_cast<unsigned long long *>(c->cv_counter.as<char>() + 16);
  double *lik_dev = c->cv_out.as<double>();
  double *lsq_dev = lik_dev + nout;
  const int *pbeg = c->cv_parts.as<int>();
  const int *pcnt = pbeg + n_sets;

  // ---- one persistent launch + finalisation, captured in a CUDA graph -------
  const size_t smem = cv_smem_bytes();
  CUDA_TRY(c, cudaFuncSetAttribute(k_cv_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
  const std::vector<uint64_t> key = {
      (uint64_t)(uintptr_t)a.x, (uint64_t)(uintptr_t)a.cell_start, (uint64_t)(uintptr_t)a.items,
      (uint64_t)(uintptr_t)a.epan_part, (uint64_t)(uintptr_t)a.conv_hist,
      (uint64_t)(uintptr_t)lik_dev, (uint64_t)a.n_items, (uint64_t)n_sets, (uint64_t)n_hx,
      (uint64_t)n_hy, (uint64_t)(uintptr_t)c->stream,
      (uint64_t)(uintptr_t)a.lutx, (uint64_t)basex, (uint64_t)basey, (uint64_t)lut_shift};
  auto enqueue = [&]() -> cudaError_t {
    cudaError_t e = cudaMemsetAsync(a.counter, 0, 32, c->stream);   // work counter + pairs
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(a.conv_hist, 0, (size_t)n_sets * 16 * kCvCells * sizeof(double),
                        c->stream);
    if (e != cudaSuccess) return e;
    k_cv_batch<<<c->sm_count, kCvBlock, smem, c->stream>>>(a);
    k_cv_finalize<<<n_sets, kCvBlock, 0, c->stream>>>(a, pbeg, pcnt, lik_dev, lsq_dev);
    return cudaGetLastError();
  };
  const bool capturable = c->stream != nullptr && c->stream != cudaStreamLegacy;
  if (capturable && (c->cv_graph == nullptr || c->cv_graph_key != key)) {
    if (c->cv_graph) { cudaGraphExecDestroy(c->cv_graph); c->cv_graph = nullptr; }
    cudaGraph_t g = nullptr;
    CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue();
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return fail(c, BBKDE_CUDA_ERROR, std::string("cv_batch graph capture: ") +
                                           cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    e = cudaGraphInstantiate(&c->cv_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      c->cv_graph = nullptr;
      return fail(c, BBKDE_CUDA_ERROR, std::string("cudaGraphInstantiate: ") +
                                           cudaGetErrorString(e));
    }
    c->cv_graph_key = key;
  }
  CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
  if (capturable) {
    CUDA_TRY(c, cudaGraphLaunch(c->cv_graph, c->stream));
  } else {
    CUDA_TRY(c, enqueue());
  }
  CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
  c->launch_total += 2;
  CUDA_TRY(c, cudaMemcpyAsync(lik_out, lik_dev, nout * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(lsq_out, lsq_dev, nout * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  unsigned long long counts[2] = {0, 0};
  CUDA_TRY(c, cudaMemcpyAsync(counts, a.pairs, sizeof(counts), cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  c->last_ms = ms;
  c->last_pairs = sum_pairs;
  c->last_launches = 2;
  c->cv_counts[0] = (int64_t)counts[0];
  c->cv_counts[1] = (int64_t)(counts[1] / 4);   // each x-power group counts every pair
  c->cv_last_plan = plan_id;
  if (trials) (*trials)[plan_id] = ms;
  return BBKDE_OK;
}

extern "C" int bbkde_cv_batch_info(const bbkde_ctx *c, int64_t *lik_pairs, int64_t *conv_pairs,
                                   int *plan, int *n_plans) {
  if (!c) return BBKDE_INVALID_ARGUMENT;
  if (lik_pairs) *lik_pairs = c->cv_counts[0];
  if (conv_pairs) *conv_pairs = c->cv_counts[1];
  if (plan) *plan = c->cv_last_plan;
  if (n_plans) *n_plans = kCvNumPlans;
  return BBKDE_OK;
}

extern "C" int bbkde_ctx_set_cv_plan(bbkde_ctx *c, int plan) {
  TRY(check_ctx(c));
  if (plan < -1 || plan >= kCvNumPlans)
    return fail(c, BBKDE_INVALID_ARGUMENT, "cv plan out of range");
  c->cv_forced_plan = plan;
  return BBKDE_OK;
}

// ===========================================================================
// Culled direct evaluation (bbkde_eval_culled) and dense grids (bbkde_eval_grid)
// ===========================================================================
namespace bbkde {
int surrogate_infer(bbkde_surrogate *s, cudaStream_t st, int64_t n, const float2 *xy,
                    int64_t gnx, double gx0, double gdx, double gy0, double gdy, float *out);
int surrogate_device(const bbkde_surrogate *s);
int surrogate_check(bbkde_surrogate *s);
}  // namespace bbkde

namespace {

// Near-field width of the culled sum in log2 units: the first pass sums every
// tile whose bound is within 2^-24 of the block's largest.
constexpr float kCullCut = 24.0f;

// Automatic probe set of the grid pipeline (bbkde_grid_config.probes = 0): 5 probes
// while the tile span is at most this many narrowest kernel widths, else 9.
constexpr double kGridProbeSpan = 0.75;
// Automatic lattice tile (bbkde_grid_config.lattice_tile = 0): 32 while a 32-point
// lattice tile spans at most this many narrowest kernel widths, else 16. The
// 32-point tile halves the kernel factors per point (1.44x the pairs per second);
// its larger box adds the references near its edge, which costs more than that
// saves on coarse lattices (measured on the Gaussian mixture: a 32-point tile of
// 10 narrowest widths 20% faster, of 33 and 80 widths 5-7% slower).
constexpr double kGridLatticeSpan = 16.0;

// Morton order of n points (x[i * stride], y[i * stride]; y null for 1-D):
// *perm_out = the sorted permutation (valid until the next sort).
int morton_sort(bbkde_ctx *c, const float *x, const float *y, int stride, int64_t n,
                const int **perm_out) {
  if (n > INT32_MAX) return fail(c, BBKDE_OUT_OF_RANGE, "more than 2^31 - 1 points");
  TRY(ensure(c, c->ms_keys, (size_t)n * sizeof(unsigned)));
  TRY(ensure(c, c->ms_keys2, (size_t)n * sizeof(unsigned)));
  TRY(ensure(c, c->ms_perm, (size_t)n * sizeof(int)));
  TRY(ensure(c, c->ms_perm2, (size_t)n * sizeof(int)));
  TRY(ensure(c, c->ms_box, 4 * sizeof(unsigned)));
  CUDA_TRY(c, cudaMemsetAsync(c->ms_box.p, 0xff, 2 * sizeof(unsigned), c->stream));
  CUDA_TRY(c, cudaMemsetAsync(c->ms_box.as<unsigned>() + 2, 0, 2 * sizeof(unsigned), c->stream));
  const unsigned gb = std::min<unsigned>(grid1d(n), (unsigned)c->sm_count * 8);
  k_bbox<<<gb, 256, 0, c->stream>>>(x, y, stride, n, c->ms_box.as<unsigned>());
  COUNT_LAUNCH(c);
  k_morton<<<grid1d(n), 256, 0, c->stream>>>(x, y, stride, n, c->ms_box.as<unsigned>(),
                                             c->ms_keys.as<unsigned>(), c->ms_perm.as<int>());
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  size_t tmp = 0;
  CUDA_TRY(c, cub::DeviceRadixSort::SortPairs(nullptr, tmp, c->ms_keys.as<unsigned>(),
                                              c->ms_keys2.as<unsigned>(), c->ms_perm.as<int>(),
                                              c->ms_perm2.as<int>(), (int)n, 0, 32, c->stream));
  TRY(ensure(c, c->ms_tmp, tmp));
  CUDA_TRY(c, cub::DeviceRadixSort::SortPairs(c->ms_tmp.p, tmp, c->ms_keys.as<unsigned>(),
                                              c->ms_keys2.as<unsigned>(), c->ms_perm.as<int>(),
                                              c->ms_perm2.as<int>(), (int)n, 0, 32, c->stream));
  c->launch_total += 4;   // CUB's onesweep radix sort: histogram + passes
  *perm_out = c->ms_perm2.as<int>();
  return BBKDE_OK;
}

// Sorted records and culling tiles of the reference set for `r` (cached).
int ensure_culled(bbkde_ctx *c, const Resolved &r) {
  TRY(ensure_pack(c, r, false));
  CullCache &cc = c->cull;
  if (cc.key == c->pack32.key) return BBKDE_OK;
  const int64_t n = c->sets[BBKDE_REFERENCE].n;
  cc.n_tiles = (int)((n + kRefTile - 1) / kRefTile);
  cc.n_groups = (cc.n_tiles + kGroupTiles - 1) / kGroupTiles;
  if (n > 0) {
    TRY(ensure(c, cc.rec, (size_t)n * sizeof(float4)));
    TRY(ensure(c, cc.ext, (size_t)n * sizeof(float)));
    TRY(ensure(c, cc.tiles, (size_t)cc.n_tiles * sizeof(RefTile)));
    TRY(ensure(c, cc.groups, (size_t)cc.n_groups * sizeof(RefTile)));
    const float *rx = c->pack32.rec.as<float>();
    const int *perm = nullptr;
    TRY(morton_sort(c, rx, r.dim == 2 ? rx + 1 : nullptr, 4, n, &perm));
    k_gather_rec<<<grid1d(n), 256, 0, c->stream>>>(c->pack32.rec.as<float4>(),
                                                   c->pack32.ext.as<float>(), perm, n,
                                                   cc.rec.as<float4>(), cc.ext.as<float>());
    COUNT_LAUNCH(c);
    const float *tex = (op_has_extra(r.op) && r.dim == 2) ? cc.ext.as<float>() : nullptr;
    const unsigned tb = grid1d((int64_t)cc.n_tiles * 32);
    if (r.dim == 2)
      k_ref_tiles<2><<<tb, 256, 0, c->stream>>>(cc.rec.as<float4>(), tex, n, cc.n_tiles,
                                                cc.tiles.as<RefTile>());
    else
      k_ref_tiles<1><<<tb, 256, 0, c->stream>>>(cc.rec.as<float4>(), tex, n, cc.n_tiles,
                                                cc.tiles.as<RefTile>());
    COUNT_LAUNCH(c);
    k_ref_groups<<<grid1d(cc.n_groups), 256, 0, c->stream>>>(
        cc.tiles.as<RefTile>(), cc.n_tiles, cc.n_groups, cc.groups.as<RefTile>());
    COUNT_LAUNCH(c);
    CUDA_TRY(c, cudaGetLastError());
  }
  cc.key = c->pack32.key;
  return BBKDE_OK;
}

// Launch shapes of the culled sum: 0 = 1024 queries per block (128 threads x 8),
// 1 = 256 queries per block (64 threads x 4).
constexpr int kCullQpb[2] = {1024, 256};

template <int OP, int D>
void launch_cull_op(int shape, unsigned nblk, cudaStream_t st, const CullArgs &a) {
  if (shape == 0)
    k_pair_sum_culled<OP, D, 8, 128, 4><<<nblk, 128, 0, st>>>(a);
  else
    k_pair_sum_culled<OP, D, 4, 64, 8><<<nblk, 64, 0, st>>>(a);
}

// Tile-16 lists shorter than this many tiles per SM are split: each tile's
// reference groups are shared by a cluster of 2, 4 or 8 blocks (the resident
// tile-16 blocks per SM: 12 by shared memory; 16-block clusters measured slower:
// 1.57 vs 1.31 ms on the 8192^2 fallback).
constexpr int kSepResidentPerSm = 12;

template <int OP, int S>
cudaError_t launch_cull_sep_split(unsigned nblk, cudaStream_t st, const CullArgs &a) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nblk * S);
  cfg.blockDim = dim3(16 * 16 / 8);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = S;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_pair_sum_culled_sep<OP, 16, S>, a);
}

// Tensor-core form of the tile-32 factored sum: the dynamic shared memory it
// requests (beyond its static arrays) keeps four blocks per SM, which together
// hold all 512 tensor-memory columns. The attribute is set on every launch, for
// the device that is current (function attributes are per device). Lists of at
// least kSepTcMinWaves waves run 128-thread blocks, shorter ones 256-thread
// blocks (the same values bitwise).
template <int OP, int NT>
cudaError_t launch_cull_sep_tc_nt(unsigned nblk, cudaStream_t st, const CullArgs &a) {
  const cudaError_t attr = cudaFuncSetAttribute(
      k_pair_sum_culled_sep_tc<OP, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
      kSepTcPadBytes);
  if (attr != cudaSuccess) return attr;
  k_pair_sum_culled_sep_tc<OP, NT><<<nblk, NT, kSepTcPadBytes, st>>>(a);
  return cudaGetLastError();
}
template <int OP>
cudaError_t launch_cull_sep_tc(unsigned nblk, cudaStream_t st, const CullArgs &a,
                               bool long_list) {
  return long_list ? launch_cull_sep_tc_nt<OP, kSepTcLongThreads>(nblk, st, a)
                   : launch_cull_sep_tc_nt<OP, kSepTcShortThreads>(nblk, st, a);
}

// parts = 1: one block per tile; 2, 4, 8 (tile 16 only): clusters of that many.
// tc: tile 32 on the tensor cores (k_pair_sum_culled_sep_tc).
template <int OP>
cudaError_t launch_cull_sep(int tile, int parts, unsigned nblk, cudaStream_t st,
                            const CullArgs &a, bool tc = false, bool long_list = false) {
  if (tile == 32 && tc) return launch_cull_sep_tc<OP>(nblk, st, a, long_list);
  if (tile == 32) {
    k_pair_sum_culled_sep<OP, 32><<<nblk, 32 * 32 / 8, 0, st>>>(a);
    return cudaGetLastError();
  }
  switch (parts) {
    case 2: return launch_cull_sep_split<OP, 2>(nblk, st, a);
    case 4: return launch_cull_sep_split<OP, 4>(nblk, st, a);
    case 8: return launch_cull_sep_split<OP, 8>(nblk, st, a);
    default:
      k_pair_sum_culled_sep<OP, 16><<<nblk, 16 * 16 / 8, 0, st>>>(a);
      return cudaGetLastError();
  }
}

// Resident factored blocks per SM: 4 at tile 32 (registers), 12 at tile 16.
int sep_resident(int tile) { return tile == 32 ? 4 : kSepResidentPerSm; }

// Reach (log2 units) of the launch-order cost proxy of factored tiles: the
// groups within 2^-32 of a tile's largest group bound.
constexpr float kSepCostReach = 32.0f;

template <int OP>
int sep_schedule(bbkde_ctx *c, CullArgs &a, unsigned nblk) {
  TRY(ensure(c, c->cb_key, (size_t)nblk * sizeof(unsigned)));
  TRY(ensure(c, c->cb_key2, (size_t)nblk * sizeof(unsigned)));
  TRY(ensure(c, c->cb_sched, (size_t)nblk * sizeof(int)));
  k_sep_tile_cost<OP><<<(unsigned)((nblk * 32 + 255) / 256), 256, 0, c->stream>>>(
      a, (int64_t)nblk, kSepCostReach, c->cb_key.as<unsigned>());
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  size_t tmp = 0;
  CUDA_TRY(c, cub::DeviceRadixSort::SortPairs(nullptr, tmp, c->cb_key.as<unsigned>(),
                                              c->cb_key2.as<unsigned>(), a.q.tile_list,
                                              c->cb_sched.as<int>(), (int)nblk, 0, 32,
                                              c->stream));
  TRY(ensure(c, c->ms_tmp, tmp));
  CUDA_TRY(c, cub::DeviceRadixSort::SortPairs(c->ms_tmp.p, tmp, c->cb_key.as<unsigned>(),
                                              c->cb_key2.as<unsigned>(), a.q.tile_list,
                                              c->cb_sched.as<int>(), (int)nblk, 0, 32,
                                              c->stream));
  c->launch_total += 4;
  a.q.tile_list = c->cb_sched.as<int>();
  return BBKDE_OK;
}

// Parts per tile for a factored launch of nblk tiles of edge `tile`.
int sep_parts(const bbkde_ctx *c, int tile, unsigned nblk) {
  if (tile != 16) return 1;
  const double per = (double)c->sm_count * kSepResidentPerSm / (double)nblk;
  return per >= 8 ? 8 : per >= 4 ? 4 : per >= 2 ? 2 : 1;
}

// One culled (or, with full, complete) sum over nblk query blocks; adds its
// statistics (pairs at tile granularity, worst bound ratio) to *pairs, *ratio.
// sep_tile > 0: grid-tile blocks of sep_tile^2 points in the factored form
// (k_pair_sum_culled_sep); the operator must factor over the axes.
// abs_n > 0 adds an absolute allowance (unnormalised units): a query's skipped
// part stays below max(rel * S, abs_n) / 2, and *ratio is then the worst skipped
// bound over that allowance; with abs_n = 0 it is the worst bound over S.
// sep_tc: a tile-32 factored sum runs on the tensor cores (k_pair_sum_culled_sep_tc).
int launch_culled(bbkde_ctx *c, const Resolved &r, int shape, unsigned nblk,
                  const CullQueries &q, double rel, bool full, double *pairs, double *ratio,
                  int sep_tile = 0, double abs_n = 0.0, bool sep_tc = false) {
  if (nblk == 0) return BBKDE_OK;
  TRY(ensure(c, c->cb_bound, (size_t)nblk * sizeof(double)));
  TRY(ensure(c, c->cb_smin, (size_t)nblk * sizeof(double)));
  TRY(ensure(c, c->cb_tiles, (size_t)nblk * sizeof(int)));
  TRY(ensure(c, c->cb_stats, 3 * sizeof(double)));   // [2]: status word of the launch
  const bool tc = sep_tc && sep_tile == 32;
  const bool tc_long =
      tc && (int64_t)nblk >= (int64_t)kSepTcMinWaves * kSepTcResident * c->sm_count;
  CullArgs a;
  a.refs = c->cull.rec.as<float4>();
  a.extra = c->cull.ext.as<float>();
  a.tiles = c->cull.tiles.as<RefTile>();
  a.groups = c->cull.groups.as<RefTile>();
  a.n_tiles = c->cull.n_tiles;
  a.n_groups = c->cull.n_groups;
  a.n_ref = c->sets[BBKDE_REFERENCE].n;
  a.cut = full ? INFINITY : kCullCut;
  a.rel = rel;
  a.abs_n = abs_n;
  a.q = q;
  a.blk_bound = c->cb_bound.as<double>();
  a.blk_smin = c->cb_smin.as<double>();
  a.blk_tiles = c->cb_tiles.as<int>();
  a.status = reinterpret_cast<int *>(c->cb_stats.as<double>() + 2);
  if (tc) CUDA_TRY(c, cudaMemsetAsync(a.status, 0, sizeof(int), c->stream));
  const bool d2 = r.dim == 2;
  if (sep_tile > 0) {
    const int parts = sep_parts(c, sep_tile, nblk);
    // More than one wave: launch the tiles most expensive first.
    if (parts == 1 && q.mode == 1 &&
        (int64_t)nblk > (int64_t)c->sm_count * sep_resident(sep_tile)) {
      switch (r.op) {
        case OP_GAUSS_ISO: TRY(sep_schedule<OP_GAUSS_ISO>(c, a, nblk)); break;
        case OP_GAUSS_PROD: TRY(sep_schedule<OP_GAUSS_PROD>(c, a, nblk)); break;
        case OP_EPAN_PROD: TRY(sep_schedule<OP_EPAN_PROD>(c, a, nblk)); break;
        default: break;
      }
    }
    switch (r.op) {
      case OP_GAUSS_ISO:
        CUDA_TRY(c, launch_cull_sep<OP_GAUSS_ISO>(sep_tile, parts, nblk, c->stream, a, tc,
                                              tc_long));
        break;
      case OP_GAUSS_PROD:
        CUDA_TRY(c, launch_cull_sep<OP_GAUSS_PROD>(sep_tile, parts, nblk, c->stream, a, tc,
                                              tc_long));
        break;
      case OP_EPAN_PROD:
        CUDA_TRY(c, launch_cull_sep<OP_EPAN_PROD>(sep_tile, parts, nblk, c->stream, a, tc,
                                              tc_long));
        break;
      default: return fail(c, BBKDE_UNSUPPORTED, "culled sum: kernel does not factor");
    }
  } else switch (r.op) {
    case OP_GAUSS_ISO:
      d2 ? launch_cull_op<OP_GAUSS_ISO, 2>(shape, nblk, c->stream, a)
         : launch_cull_op<OP_GAUSS_ISO, 1>(shape, nblk, c->stream, a);
      break;
    case OP_GAUSS_PROD: launch_cull_op<OP_GAUSS_PROD, 2>(shape, nblk, c->stream, a); break;
    case OP_EPAN_ISO:
      d2 ? launch_cull_op<OP_EPAN_ISO, 2>(shape, nblk, c->stream, a)
         : launch_cull_op<OP_EPAN_ISO, 1>(shape, nblk, c->stream, a);
      break;
    case OP_EPAN_PROD: launch_cull_op<OP_EPAN_PROD, 2>(shape, nblk, c->stream, a); break;
    default: return fail(c, BBKDE_UNSUPPORTED, "culled sum: unsupported kernel");
  }
  COUNT_LAUNCH(c);
  k_cull_stats<<<1, 256, 0, c->stream>>>(a.blk_bound, a.blk_smin, a.blk_tiles, (int)nblk,
                                         c->cb_stats.as<double>());
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  double st[3];
  CUDA_TRY(c, cudaMemcpyAsync(st, c->cb_stats.p, (tc ? 3 : 2) * sizeof(double),
                              cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (tc) {
    int status = 0;
    std::memcpy(&status, &st[2], sizeof(int));
    if (status != 0)
      return fail(c, BBKDE_CUDA_ERROR,
                  "culled sum: a tensor-core wait expired (the results are not written)");
  }
  if (pairs) *pairs += st[1] * kRefTile * kCullQpb[shape];
  if (ratio) *ratio = std::max(*ratio, abs_n > 0.0 ? st[0] : st[0] * rel);
  return BBKDE_OK;
}

int culled_kernel_ok(bbkde_ctx *c, const Resolved &r) {
  if (r.op == OP_EPAN_CONV)
    return fail(c, BBKDE_UNSUPPORTED,
                "culled sum: the Epanechnikov convolution kernels are not supported");
  return BBKDE_OK;
}

}  // namespace

namespace {

// The culled evaluation of the QUERY set with a relative tolerance rel and an
// absolute one abs_err (normalised density units, as the reference's abs_err).
int eval_culled_impl(bbkde_ctx *c, const bbkde_kernel_desc *k, int normalized, double rel_tol,
                     double abs_err, double *out, int out_on_device, bbkde_cull_stats *stats) {
  Resolved r;
  TRY(resolve(c, k, r));
  TRY(culled_kernel_ok(c, r));
  // the tree scales abs_err by 1 / C(h) for its unnormalised sums (:723-729)
  const double abs_n = abs_err > 0.0 ? abs_err / r.norm : 0.0;
  const PointSet &rs = c->sets[BBKDE_REFERENCE], &qs = c->sets[BBKDE_QUERY];
  if ((rs.n > 0 && rs.dim != r.dim) || (qs.n > 0 && qs.dim != r.dim))
    return fail(c, BBKDE_INVALID_ARGUMENT, "point dimension does not match the kernel");
  bbkde_cull_stats st = {0.0, 0.0, (double)rs.n * (double)qs.n, 0.0};
  const int64_t nq = qs.n;
  if (nq == 0) {
    if (stats) *stats = st;
    return BBKDE_OK;
  }
  double *dst = out;
  if (!out_on_device) {
    TRY(ensure(c, c->out_dev, (size_t)nq * sizeof(double)));
    dst = c->out_dev.as<double>();
  }
  if (rs.n == 0) {
    CUDA_TRY(c, cudaMemsetAsync(dst, 0, (size_t)nq * sizeof(double), c->stream));
  } else {
    TRY(ensure_culled(c, r));
    const void *qx = nullptr, *qy = nullptr;
    TRY(ensure_queries(c, BBKDE_QUERY, false, &qx, &qy));
    const float *fx = static_cast<const float *>(qx), *fy = static_cast<const float *>(qy);
    const int *perm = nullptr;
    TRY(morton_sort(c, fx, r.dim == 2 ? fy : nullptr, 1, nq, &perm));
    TRY(ensure(c, c->cq_x, (size_t)nq * sizeof(float)));
    TRY(ensure(c, c->cq_y, (size_t)nq * sizeof(float)));
    TRY(ensure(c, c->cq_out, (size_t)nq * sizeof(double)));
    k_gather_xy<<<grid1d(nq), 256, 0, c->stream>>>(fx, r.dim == 2 ? fy : nullptr, perm, nq,
                                                   c->cq_x.as<float>(), c->cq_y.as<float>());
    COUNT_LAUNCH(c);
    CullQueries q = {};
    q.mode = 0;
    q.qx = c->cq_x.as<float>();
    q.qy = c->cq_y.as<float>();
    q.count = nq;
    q.out = c->cq_out.as<double>();
    q.scale = normalized ? r.norm : 1.0;
    const unsigned nblk = (unsigned)((nq + kCullQpb[0] - 1) / kCullQpb[0]);
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    TRY(launch_culled(c, r, 0, nblk, q, rel_tol, false, &st.pairs, &st.max_bound_ratio, 0,
                      abs_n));
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    k_scatter<<<grid1d(nq), 256, 0, c->stream>>>(c->cq_out.as<double>(), perm, nq, dst);
    COUNT_LAUNCH(c);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    st.kernel_ms = ms;
  }
  if (!out_on_device)
    CUDA_TRY(c, cudaMemcpyAsync(out, dst, (size_t)nq * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->last_ms = st.kernel_ms;
  c->last_pairs = st.pairs;
  c->last_launches = 2;
  if (stats) *stats = st;
  return BBKDE_OK;
}

}  // namespace

extern "C" int bbkde_eval_culled(bbkde_ctx *c, const bbkde_kernel_desc *k, int normalized,
                                 double rel_tol, double *out, int out_on_device,
                                 bbkde_cull_stats *stats) {
  TRY(check_ctx(c));
  if (!out) return fail(c, BBKDE_INVALID_ARGUMENT, "output pointer is NULL");
  if (!(rel_tol > 0.0 && rel_tol < 1.0))
    return fail(c, BBKDE_INVALID_ARGUMENT, "rel_tol must be in (0, 1)");
  return eval_culled_impl(c, k, normalized, rel_tol, 0.0, out, out_on_device, stats);
}

extern "C" int bbkde_eval_tol(bbkde_ctx *c, const bbkde_kernel_desc *k, int normalized,
                              double rel_err, double abs_err, double *out, int out_on_device,
                              bbkde_cull_stats *stats) {
  TRY(check_ctx(c));
  if (!out) return fail(c, BBKDE_INVALID_ARGUMENT, "output pointer is NULL");
  if (!(rel_err >= 0.0 && rel_err < 1.0) || !(abs_err >= 0.0) || !std::isfinite(abs_err))
    return fail(c, BBKDE_INVALID_ARGUMENT,
                "need 0 <= rel_err < 1 and a finite abs_err >= 0");
  return eval_culled_impl(c, k, normalized, rel_err, abs_err, out, out_on_device, stats);
}

namespace {

// Normalised culled self-sum of the REFERENCE set with its current attributes,
// self term included: out[i] (device, the set's order) within max(rel * f_i,
// abs_err) / 2 of f_i = C sum_j m_j U(x_i, x_j) (abs_err in normalised density
// units), FP32-compensated. Queries are the set's own FP32
// coordinates in Morton order. *pairs gets the pairs at tile granularity and
// *ms the device time of the culled launch.
int culled_self_sum(bbkde_ctx *c, const Resolved &r, double rel, double abs_err, double *out,
                    double *pairs, float *ms) {
  const int64_t n = c->sets[BBKDE_REFERENCE].n;
  TRY(ensure_culled(c, r));
  const void *qx = nullptr, *qy = nullptr;
  TRY(ensure_queries(c, BBKDE_REFERENCE, false, &qx, &qy));
  const float *fx = static_cast<const float *>(qx), *fy = static_cast<const float *>(qy);
  const int *perm = nullptr;
  TRY(morton_sort(c, fx, r.dim == 2 ? fy : nullptr, 1, n, &perm));
  TRY(ensure(c, c->cq_x, (size_t)n * sizeof(float)));
  TRY(ensure(c, c->cq_y, (size_t)n * sizeof(float)));
  TRY(ensure(c, c->cq_out, (size_t)std::max<int64_t>(n, kWlogBlocks) * sizeof(double)));
  k_gather_xy<<<grid1d(n), 256, 0, c->stream>>>(fx, r.dim == 2 ? fy : nullptr, perm, n,
                                                c->cq_x.as<float>(), c->cq_y.as<float>());
  COUNT_LAUNCH(c);
  CullQueries q = {};
  q.mode = 0;
  q.qx = c->cq_x.as<float>();
  q.qy = c->cq_y.as<float>();
  q.count = n;
  q.out = c->cq_out.as<double>();
  q.scale = r.norm;
  double ratio = 0.0;
  *pairs = 0.0;
  CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
  TRY(launch_culled(c, r, 0, (unsigned)((n + kCullQpb[0] - 1) / kCullQpb[0]), q, rel, false,
                    pairs, &ratio, 0, abs_err > 0.0 ? abs_err / r.norm : 0.0));
  CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
  k_scatter<<<grid1d(n), 256, 0, c->stream>>>(c->cq_out.as<double>(), perm, n, out);
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  CUDA_TRY(c, cudaEventSynchronize(c->ev1));
  CUDA_TRY(c, cudaEventElapsedTime(ms, c->ev0, c->ev1));
  return BBKDE_OK;
}

// FP64 sum over the set of w_i log(f_i - sub_i C) (mode 0) or w_i (f_i - sub_i C)
// (mode 1), sub = null for no subtraction, in fixed order -> *dst (device).
int wsum(bbkde_ctx *c, const double *f, const double *sub, double C, int mode, int64_t n,
         double *dst) {
  TRY(ensure(c, c->cq_out, (size_t)std::max<int64_t>(n, kWlogBlocks) * sizeof(double)));
  k_wsum_partial<<<kWlogBlocks, 256, 0, c->stream>>>(
      f, sub, C, c->sets[BBKDE_REFERENCE].weight.as<double>(), mode, n, c->cq_out.as<double>());
  COUNT_LAUNCH(c);
  k_sum_partials<<<1, kWlogBlocks, 0, c->stream>>>(c->cq_out.as<double>(), kWlogBlocks, dst);
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  return BBKDE_OK;
}

// Argument checks of the tolerance forms: 0 <= rel_tol < 1, finite abs_tol >= 0
// (both 0: every tile that does not flush to zero is summed).
int tol_checks(bbkde_ctx *c, const bbkde_kernel_desc *k, double rel_tol, double abs_tol,
               Resolved &r) {
  TRY(self_checks(c, k, BBKDE_FP32C, r));
  TRY(culled_kernel_ok(c, r));
  if (!(rel_tol >= 0.0 && rel_tol < 1.0) || !(abs_tol >= 0.0) || !std::isfinite(abs_tol))
    return fail(c, BBKDE_INVALID_ARGUMENT,
                "tolerances: need 0 <= rel_tol < 1 and a finite abs_tol >= 0");
  return BBKDE_OK;
}

}  // namespace

// Adaptive densities with the pilot to a tolerance (KernelDensity::adapt_density
// (alpha, rel, abs), KernelDensityImpl.h:291-359, whose pilot the reference
// evaluates through its tree to rel / abs): the pilot is the culled self-sum of
// the reference set (every value within max(rel_tol f, abs_tol) / 2 of the full
// sum f, self term included, FP32-compensated), the rest is
// bbkde_adapt_density's FP64 epilogue.
extern "C" int bbkde_adapt_density_tol(bbkde_ctx *c, const bbkde_kernel_desc *k, double alpha,
                                       double rel_tol, double abs_tol, double *abw_out,
                                       double *mass_out, double *pilot_out, double *g_out) {
  Resolved r;
  TRY(tol_checks(c, k, rel_tol, abs_tol, r));
  if (!(alpha >= 0 && alpha <= 1))   // KernelDensityImpl.h:301-303
    return fail(c, BBKDE_INVALID_ARGUMENT, "adapt_density: alpha must be between [0, 1]. ");
  TRY(bbkde_unadapt_density(c));
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (alpha == 0 || s.n == 0) {
    if (g_out) *g_out = NAN;
    TRY(download(c, abw_out, s.abw, s.n));
    TRY(download(c, mass_out, s.mass, s.n));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return BBKDE_OK;
  }
  const int64_t n = s.n;
  TRY(ensure(c, c->out_dev, (size_t)n * sizeof(double)));
  double *pilot = c->out_dev.as<double>();
  double pairs = 0.0;
  float ms = 0.f;
  TRY(culled_self_sum(c, r, rel_tol, abs_tol, pilot, &pairs, &ms));
  // g = exp(sum_i w_i log pilot_i) in FP64, fixed order (:330-337).
  TRY(wsum(c, pilot, nullptr, 0.0, 0, n, c->scalars.as<double>()));
  k_pilot_finalize<<<grid1d(n), 256, 0, c->stream>>>(
      pilot, s.weight.as<double>(), c->scalars.as<double>(), alpha, r.dim, n,
      s.abw.as<double>(), s.mass.as<double>(), c->scalars.as<double>() + 1);
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  ++s.attr_version;
  TRY(download(c, pilot_out, c->out_dev, n));
  TRY(download(c, abw_out, s.abw, n));
  TRY(download(c, mass_out, s.mass, n));
  double g = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&g, c->scalars.as<double>() + 1, sizeof(double),
                              cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (g_out) *g_out = g;
  c->last_ms = ms;
  c->last_pairs = pairs;
  c->last_launches = 6;
  return BBKDE_OK;
}

// Cross validation with the density sums to a tolerance, as the reference
// evaluates them through its tree (likelihood_cross_validate,
// KernelDensityImpl.h:215-252; lsq_convolution_cross_validate, :142-209): the
// full self-sums are culled sums within max(rel_tol f, abs_tol) / 2, and the
// leave-one-out value is the full sum minus the self term m_i C(h), as the
// reference computes it.
extern "C" int bbkde_likelihood_cv_tol(bbkde_ctx *c, const bbkde_kernel_desc *k, double rel_tol,
                                       double abs_tol, double *cv_out) {
  Resolved r;
  TRY(tol_checks(c, k, rel_tol, abs_tol, r));
  if (!cv_out) return fail(c, BBKDE_INVALID_ARGUMENT, "cv_out is NULL");
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (s.n == 0) { *cv_out = 0.0; return BBKDE_OK; }
  TRY(ensure(c, c->out_dev, (size_t)s.n * sizeof(double)));
  double pairs = 0.0;
  float ms = 0.f;
  TRY(culled_self_sum(c, r, rel_tol, abs_tol, c->out_dev.as<double>(), &pairs, &ms));
  // sum_i w_i log(f_i - m_i C) (:240-249)
  TRY(wsum(c, c->out_dev.as<double>(), s.mass.as<double>(), r.norm, 0, s.n,
           c->scalars.as<double>()));
  CUDA_TRY(c, cudaMemcpyAsync(cv_out, c->scalars.p, sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->last_ms = ms;
  c->last_pairs = pairs;
  return BBKDE_OK;
}

extern "C" int bbkde_lsq_conv_cv_tol(bbkde_ctx *c, const bbkde_kernel_desc *k, double rel_tol,
                                     double abs_tol, double *cv_out) {
  Resolved r;
  TRY(tol_checks(c, k, rel_tol, abs_tol, r));
  if (!cv_out) return fail(c, BBKDE_INVALID_ARGUMENT, "cv_out is NULL");
  const int ck = conv_kind_of(k->kind, k->dim);
  if (ck < 0)
    return fail(c, BBKDE_UNSUPPORTED, "no convolution kernel is associated with this kernel");
  bbkde_kernel_desc kc = *k;
  kc.kind = ck;
  Resolved rc;
  TRY(resolve(c, &kc, rc));
  TRY(culled_kernel_ok(c, rc));
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (s.n == 0) { *cv_out = 0.0; return BBKDE_OK; }
  TRY(ensure(c, c->out_dev, (size_t)s.n * sizeof(double)));
  double pairs = 0.0, pairs2 = 0.0;
  float ms = 0.f, ms2 = 0.f;
  double t[2];
  // Leave-one-out term sum_i w_i (f_i - m_i C) (:162-181).
  TRY(culled_self_sum(c, r, rel_tol, abs_tol, c->out_dev.as<double>(), &pairs, &ms));
  TRY(wsum(c, c->out_dev.as<double>(), s.mass.as<double>(), r.norm, 1, s.n,
           c->scalars.as<double>()));
  // Square-integral term sum_i w_i f_conv(x_i), self term included (:187-205).
  TRY(culled_self_sum(c, rc, rel_tol, abs_tol, c->out_dev.as<double>(), &pairs2, &ms2));
  TRY(wsum(c, c->out_dev.as<double>(), nullptr, 0.0, 1, s.n, c->scalars.as<double>() + 1));
  CUDA_TRY(c, cudaMemcpyAsync(t, c->scalars.p, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  *cv_out = t[1] - 2.0 * t[0];   // :207
  c->last_ms = ms + ms2;
  c->last_pairs = pairs + pairs2;
  return BBKDE_OK;
}

namespace {

// Tile numbers of g in Morton order of their coordinates -> order (ntiles ints).
int tile_order(bbkde_ctx *c, const GridDesc &g, DevBuf &order) {
  const int64_t nt = (int64_t)g.ntx * g.nty;
  TRY(ensure(c, c->ms_keys, (size_t)nt * sizeof(unsigned)));
  TRY(ensure(c, c->ms_keys2, (size_t)nt * sizeof(unsigned)));
  TRY(ensure(c, c->ms_perm, (size_t)nt * sizeof(int)));
  TRY(ensure(c, order, (size_t)nt * sizeof(int)));
  k_tile_keys<<<grid1d(nt), 256, 0, c->stream>>>(g, c->ms_keys.as<unsigned>(),
                                                 c->ms_perm.as<int>());
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  size_t tmp = 0;
  CUDA_TRY(c, cub::DeviceRadixSort::SortPairs(nullptr, tmp, c->ms_keys.as<unsigned>(),
                                              c->ms_keys2.as<unsigned>(), c->ms_perm.as<int>(),
                                              order.as<int>(), (int)nt, 0, 32, c->stream));
  TRY(ensure(c, c->ms_tmp, tmp));
  CUDA_TRY(c, cub::DeviceRadixSort::SortPairs(c->ms_tmp.p, tmp, c->ms_keys.as<unsigned>(),
                                              c->ms_keys2.as<unsigned>(), c->ms_perm.as<int>(),
                                              order.as<int>(), (int)nt, 0, 32, c->stream));
  c->launch_total += 4;
  return BBKDE_OK;
}

GridDesc make_grid(int64_t nx, int64_t ny, double x0, double dx, double y0, double dy, int tile) {
  GridDesc g;
  g.nx = nx;
  g.ny = ny;
  g.x0 = x0;
  g.dx = dx;
  g.y0 = y0;
  g.dy = dy;
  g.tile = tile;
  g.ntx = (int)((nx + tile - 1) / tile);
  g.nty = (int)((ny + tile - 1) / tile);
  return g;
}

// Exact sums at the points of every listed tile of g (results row-major into out),
// in the factored form where the kernel factors over the axes unless pair_form.
// tensor_cores (bbkde_grid_config.tensor_cores): 0 = tile-32 factored sums on the
// tensor cores when rel >= kSepTcMinRel (culled), 1 = never, 2 = always.
int grid_exact(bbkde_ctx *c, const Resolved &r, const GridDesc &g, const int *list, int64_t n,
               double rel, bool full, double *out, double *pairs, double *ratio,
               bool pair_form = false, int tensor_cores = 1) {
  CullQueries q = {};
  q.mode = 1;
  q.tile_list = list;
  q.tile = g.tile;
  q.ntx = g.ntx;
  q.gnx = g.nx;
  q.gny = g.ny;
  q.gx0 = g.x0;
  q.gdx = g.dx;
  q.gy0 = g.y0;
  q.gdy = g.dy;
  q.out = out;
  q.scale = r.norm;
  const int shape = g.tile == 32 ? 0 : 1;
  const int sep = (!pair_form && r.dim == 2 && op_separable(r.op)) ? g.tile : 0;
  const bool tc = sep == 32 && (tensor_cores == 2 ||
                                (tensor_cores == 0 && !full && rel >= kSepTcMinRel));
  return launch_culled(c, r, shape, (unsigned)n, q, rel, full, pairs, ratio, sep, 0.0, tc);
}

}  // namespace

extern "C" int bbkde_eval_grid(bbkde_ctx *c, bbkde_surrogate *sur, const bbkde_kernel_desc *k,
                               const bbkde_grid *grid, const bbkde_grid_config *cfg,
                               double *out, bbkde_grid_stats *stats) {
  TRY(check_ctx(c));
  if (!grid || !cfg || !out) return fail(c, BBKDE_INVALID_ARGUMENT, "NULL argument");
  if (grid->nx < 1 || grid->ny < 1 || !(grid->x1 > grid->x0) || !(grid->y1 > grid->y0) ||
      !std::isfinite(grid->x0) || !std::isfinite(grid->x1) || !std::isfinite(grid->y0) ||
      !std::isfinite(grid->y1))
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: need nx, ny >= 1 and finite x0 < x1, y0 < y1");
  const int mode = cfg->mode, T = cfg->tile;
  int P = cfg->probes;
  if (mode < BBKDE_GRID_EXACT || mode > BBKDE_GRID_ANCHORED)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: unknown mode");
  if (T != 16 && T != 32) return fail(c, BBKDE_INVALID_ARGUMENT, "grid: tile must be 16 or 32");
  if (P != 0 && P != 1 && P != 5 && P != 9)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: probes must be 0 (automatic), 1, 5 or 9");
  int LT = cfg->lattice_tile;
  if (LT != 0 && LT != 16 && LT != 32)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: lattice_tile must be 0, 16 or 32");
  if (cfg->tensor_cores < 0 || cfg->tensor_cores > 2)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: tensor_cores must be 0, 1 or 2");
  const int interp = cfg->interp == 0 ? 1 : cfg->interp;
  if (interp != 1 && interp != 3)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: interp must be 1 (bilinear) or 3 (bicubic)");
  if (!(cfg->rel_tol > 0) || !(cfg->low_frac >= 0 && cfg->low_frac < 1) ||
      !(cfg->cull_rel > 0 && cfg->cull_rel < 1))
    return fail(c, BBKDE_INVALID_ARGUMENT,
                "grid: need rel_tol > 0, 0 <= low_frac < 1, 0 < cull_rel < 1");
  if (mode == BBKDE_GRID_SURROGATE && !sur)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: surrogate mode needs a surrogate");
  if (mode != BBKDE_GRID_EXACT && sur && bbkde::surrogate_device(sur) != c->device)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: surrogate lives on another device");
  Resolved r;
  TRY(resolve(c, k, r));
  TRY(culled_kernel_ok(c, r));
  if (r.dim != 2) return fail(c, BBKDE_INVALID_ARGUMENT, "grid: the kernel must be 2-D");
  const PointSet &rs = c->sets[BBKDE_REFERENCE];
  if (rs.n > 0 && rs.dim != 2)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: the reference set must be 2-D");
  const GridDesc g = make_grid(grid->nx, grid->ny, grid->x0, (grid->x1 - grid->x0) / grid->nx,
                               grid->y0, (grid->y1 - grid->y0) / grid->ny, T);
  if (g.ntx > 65535 || g.nty > 65535 || (int64_t)g.ntx * g.nty > (int64_t)1 << 30)
    return fail(c, BBKDE_OUT_OF_RANGE, "grid: too many tiles");
  const int64_t npts = g.nx * g.ny, ntiles = (int64_t)g.ntx * g.nty;
  const bool full = cfg->exact_culled == 0;
  if (P == 0 || LT == 0) {
    // Automatic probe set: the centre and edge midpoints suffice while a tile spans
    // at most kGridProbeSpan narrowest kernel widths (h times the smallest abw);
    // wider tiles vary between those probes, so the quarter points join them.
    // Automatic lattice tile: kGridLatticeSpan.
    double amin = 1.0;
    if (rs.n > 0 && c->abw_min_cv == rs.coord_version && c->abw_min_av == rs.attr_version) {
      amin = c->abw_min;
    } else if (rs.n > 0) {
      const unsigned nb = std::min<unsigned>(grid1d(rs.n), (unsigned)c->sm_count * 4);
      TRY(ensure(c, c->gr_part, (size_t)nb * sizeof(double)));
      k_min_positive<<<nb, 256, 0, c->stream>>>(rs.abw.as<double>(), rs.n,
                                                c->gr_part.as<double>(), false);
      k_min_positive<<<1, 1024, 0, c->stream>>>(c->gr_part.as<double>(), (int64_t)nb,
                                                c->scalars.as<double>() + 8, true);
      c->launch_total += 2;
      CUDA_TRY(c, cudaGetLastError());
      CUDA_TRY(c, cudaMemcpyAsync(&amin, c->scalars.as<double>() + 8, sizeof(double),
                                  cudaMemcpyDeviceToHost, c->stream));
      CUDA_TRY(c, cudaStreamSynchronize(c->stream));
      c->abw_min = amin;
      c->abw_min_cv = rs.coord_version;
      c->abw_min_av = rs.attr_version;
    }
    const double wmin = std::min(r.h1, r.h2) * amin;
    const double span = T * std::max(g.dx, g.dy);
    if (P == 0) P = span <= kGridProbeSpan * wmin ? 5 : 9;
    if (LT == 0) LT = 32 * (T / 2) * std::max(g.dx, g.dy) <= kGridLatticeSpan * wmin ? 32 : 16;
  }
  bbkde_grid_stats st = {};
  st.tiles = ntiles;
  st.probes_used = P;
  st.lattice_tile_used = LT;
  if (rs.n == 0) {
    CUDA_TRY(c, cudaMemsetAsync(out, 0, (size_t)npts * sizeof(double), c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    st.tiles_flagged = ntiles;
    if (stats) *stats = st;
    return BBKDE_OK;
  }
  TRY(ensure_culled(c, r));
  TRY(tile_order(c, g, c->gr_order));
  TRY(ensure(c, c->gr_flag, (size_t)ntiles * sizeof(int)));
  TRY(ensure(c, c->gr_flag_ord, (size_t)ntiles * sizeof(int)));
  TRY(ensure(c, c->gr_list, (size_t)ntiles * sizeof(int)));
  TRY(ensure(c, c->gr_nsel, sizeof(int)));
  TRY(ensure(c, c->gr_counts, 3 * sizeof(unsigned long long)));
  TRY(ensure(c, c->gr_gmax, sizeof(float)));
  TRY(ensure(c, c->gr_tmin, (size_t)ntiles * sizeof(float)));
  TRY(ensure(c, c->gr_tmax, (size_t)ntiles * sizeof(float)));
  TRY(ensure(c, c->gr_bad, (size_t)ntiles * sizeof(int)));
  TRY(ensure(c, c->gr_terr, (size_t)ntiles * sizeof(unsigned)));
  CUDA_TRY(c, cudaMemsetAsync(c->gr_counts.p, 0, 3 * sizeof(unsigned long long), c->stream));
  CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));

  FlagArgs fa;
  fa.g = g;
  fa.order = c->gr_order.as<int>();
  fa.tmin = c->gr_tmin.as<float>();
  fa.bad = c->gr_bad.as<int>();
  fa.terr = c->gr_terr.as<unsigned>();
  fa.gmax = c->gr_gmax.as<float>();
  fa.log_low = cfg->low_frac > 0 ? (float)std::log(cfg->low_frac) : -INFINITY;
  fa.rel_tol = (float)cfg->rel_tol;
  fa.all = mode == BBKDE_GRID_EXACT;
  fa.flag = c->gr_flag.as<int>();
  fa.flag_ord = c->gr_flag_ord.as<int>();
  fa.counts = c->gr_counts.as<unsigned long long>();

  // Rescue mode: the network runs after the probes, on the missed tiles only.
  const bool rescue =
      mode == BBKDE_GRID_ANCHORED && sur && cfg->net_scope != BBKDE_NET_EVERYWHERE;
  const bool net_all = mode != BBKDE_GRID_EXACT && sur && !rescue;
  if (mode == BBKDE_GRID_EXACT) {
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    CUDA_TRY(c, cudaEventRecord(c->ev2, c->stream));
    k_flag_tiles<<<grid1d(ntiles), 256, 0, c->stream>>>(fa);
    COUNT_LAUNCH(c);
  } else {
    // 1. Prediction at every point (log-density): the network, or zero.
    bool pred_zero = false;
    TRY(ensure(c, c->gr_pred, (size_t)npts * sizeof(float)));
    float *pred = c->gr_pred.as<float>();
    if (net_all) {
      TRY(bbkde::surrogate_infer(sur, c->stream, npts, nullptr, g.nx, g.x0, g.dx, g.y0, g.dy,
                                 pred) == BBKDE_OK
              ? BBKDE_OK
              : fail(c, BBKDE_CUDA_ERROR, "grid: surrogate inference failed"));
      COUNT_LAUNCH(c);
    } else {
      pred_zero = true;   // written by the interpolation below, never read as zeros
    }
    if (!rescue) CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    // 2. Exact values on the half-pitch lattice (anchors and probes; one regular
    //    grid of pitch T/2 from the grid's origin, past its end by one pitch) and,
    //    for 9 probes, on the quarter lattice; network values there.
    const int h = T / 2;
    const GridDesc gl = make_grid(2 * (int64_t)g.ntx + 1, 2 * (int64_t)g.nty + 1, g.x0,
                                  h * g.dx, g.y0, h * g.dy, LT);
    const int64_t n_lat = gl.nx * gl.ny;
    TRY(ensure(c, c->gr_lat_exact, (size_t)n_lat * sizeof(double)));
    TRY(tile_order(c, gl, c->gr_lat_order));
    TRY(grid_exact(c, r, gl, c->gr_lat_order.as<int>(), (int64_t)gl.ntx * gl.nty,
                   cfg->cull_rel, full, c->gr_lat_exact.as<double>(), &st.pairs,
                   &st.max_bound_ratio, cfg->pair_form != 0, cfg->tensor_cores));
    auto lattice_net = [&]() -> int {
      TRY(ensure(c, c->gr_lat_net, (size_t)n_lat * sizeof(float)));
      TRY(bbkde::surrogate_infer(sur, c->stream, n_lat, nullptr, gl.nx, gl.x0, gl.dx, gl.y0,
                                 gl.dy, c->gr_lat_net.as<float>()) == BBKDE_OK
              ? BBKDE_OK
              : fail(c, BBKDE_CUDA_ERROR, "grid: surrogate inference failed"));
      COUNT_LAUNCH(c);
      return BBKDE_OK;
    };
    const float *lat_net = nullptr, *q_net = nullptr;
    if (net_all) {
      TRY(lattice_net());
      lat_net = c->gr_lat_net.as<float>();
    }
    int64_t n_q = 0;
    const GridDesc gq = make_grid(2 * (int64_t)g.ntx, 2 * (int64_t)g.nty, g.x0 + (T / 4) * g.dx,
                                  h * g.dx, g.y0 + (T / 4) * g.dy, h * g.dy, LT);
    auto quarter_net = [&]() -> int {
      TRY(ensure(c, c->gr_q_net, (size_t)n_q * sizeof(float)));
      TRY(bbkde::surrogate_infer(sur, c->stream, n_q, nullptr, gq.nx, gq.x0, gq.dx, gq.y0,
                                 gq.dy, c->gr_q_net.as<float>()) == BBKDE_OK
              ? BBKDE_OK
              : fail(c, BBKDE_CUDA_ERROR, "grid: surrogate inference failed"));
      COUNT_LAUNCH(c);
      return BBKDE_OK;
    };
    if (P == 9) {
      n_q = gq.nx * gq.ny;
      TRY(ensure(c, c->gr_q_exact, (size_t)n_q * sizeof(double)));
      TRY(tile_order(c, gq, c->gr_q_order));
      TRY(grid_exact(c, r, gq, c->gr_q_order.as<int>(), (int64_t)gq.ntx * gq.nty, cfg->cull_rel,
                     full, c->gr_q_exact.as<double>(), &st.pairs, &st.max_bound_ratio,
                     cfg->pair_form != 0, cfg->tensor_cores));
      if (net_all) {
        TRY(quarter_net());
        q_net = c->gr_q_net.as<float>();
      }
    }
    // 3. Anchored mode: residual at the anchors, interpolated onto the grid.
    const int64_t n_anchor = ((int64_t)g.ntx + 1) * (g.nty + 1);
    const float *resid = nullptr;
    if (mode == BBKDE_GRID_ANCHORED) {
      TRY(ensure(c, c->gr_resid, (size_t)n_anchor * sizeof(float)));
      k_anchor_residual<<<grid1d(n_anchor), 256, 0, c->stream>>>(
          c->gr_lat_exact.as<double>(), lat_net, g.ntx, g.nty, c->gr_resid.as<float>());
      COUNT_LAUNCH(c);
      resid = c->gr_resid.as<float>();
    }
    if (pred_zero && !resid) {
      CUDA_TRY(c, cudaMemsetAsync(pred, 0, (size_t)npts * sizeof(float), c->stream));
      pred_zero = false;
    }
    k_tile_reduce<<<(unsigned)((ntiles + kTileReduceWarps - 1) / kTileReduceWarps),
                    32 * kTileReduceWarps, 0, c->stream>>>(g, pred, resid, interp, pred_zero ? 1 : 0,
                                                           c->gr_tmin.as<float>(),
                                                           c->gr_tmax.as<float>(),
                                                           c->gr_bad.as<int>());
    COUNT_LAUNCH(c);
    {
      const unsigned nb = std::min<unsigned>(grid1d(ntiles), (unsigned)c->sm_count * 4);
      TRY(ensure(c, c->gr_part, (size_t)nb * sizeof(double)));
      k_max_finite<<<nb, 256, 0, c->stream>>>(c->gr_tmax.as<float>(), (int)ntiles,
                                              c->gr_part.as<float>());
      k_max_finite<<<1, 1024, 0, c->stream>>>(c->gr_part.as<float>(), (int)nb,
                                              c->gr_gmax.as<float>());
      c->launch_total += 2;
    }
    // 4. Held-out probes: every tile's interpolant against the exact lattice values.
    ProbeArgs pa;
    pa.g = g;
    pa.list = nullptr;
    pa.n_list = 0;
    pa.lat_exact = c->gr_lat_exact.as<double>();
    pa.lat_net = lat_net;
    pa.q_exact = P == 9 ? c->gr_q_exact.as<double>() : nullptr;
    pa.q_net = q_net;
    pa.resid = resid;
    pa.interp = interp;
    pa.probes = P;
    pa.terr = c->gr_terr.as<unsigned>();
    k_probe_check<<<grid1d(ntiles), 256, 0, c->stream>>>(pa);
    COUNT_LAUNCH(c);
    k_flag_tiles<<<grid1d(ntiles), 256, 0, c->stream>>>(fa);
    COUNT_LAUNCH(c);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaEventRecord(rescue ? c->ev1 : c->ev2, c->stream));
    st.exact_points = n_lat + n_q;

    // 5. Rescue: the network + its own residual on the tiles whose probes missed;
    //    a tile keeps that prediction when its probes pass.
    if (rescue) {
      TRY(ensure(c, c->gr_cand_ord, (size_t)ntiles * sizeof(int)));
      k_rescue_mark<<<grid1d(ntiles), 256, 0, c->stream>>>(fa, c->gr_cand_ord.as<int>());
      COUNT_LAUNCH(c);
      size_t tmp = 0;
      CUDA_TRY(c, cub::DeviceSelect::Flagged(nullptr, tmp, c->gr_order.as<int>(),
                                             c->gr_cand_ord.as<int>(), c->gr_list.as<int>(),
                                             c->gr_nsel.as<int>(), (int)ntiles, c->stream));
      TRY(ensure(c, c->ms_tmp, tmp));
      CUDA_TRY(c, cub::DeviceSelect::Flagged(c->ms_tmp.p, tmp, c->gr_order.as<int>(),
                                             c->gr_cand_ord.as<int>(), c->gr_list.as<int>(),
                                             c->gr_nsel.as<int>(), (int)ntiles, c->stream));
      c->launch_total += 2;
      int ncand = 0;
      CUDA_TRY(c, cudaMemcpyAsync(&ncand, c->gr_nsel.p, sizeof(int), cudaMemcpyDeviceToHost,
                                  c->stream));
      CUDA_TRY(c, cudaStreamSynchronize(c->stream));
      if (ncand > 0) {
        const int *cand = c->gr_list.as<int>();
        // The network on the lattice points the candidates read (their anchors
        // and probes), not on the whole lattice; NaN elsewhere (read by nothing).
        const int64_t nl = (int64_t)ncand * kRescueSlots;
        TRY(ensure(c, c->gr_lat_net, (size_t)n_lat * sizeof(float)));
        TRY(ensure(c, c->gr_rl_idx, (size_t)nl * sizeof(int64_t)));
        TRY(ensure(c, c->gr_rl_xy, (size_t)nl * sizeof(float2)));
        TRY(ensure(c, c->gr_rl_net, (size_t)nl * sizeof(float)));
        CUDA_TRY(c, cudaMemsetAsync(c->gr_lat_net.p, 0xff, (size_t)n_lat * sizeof(float),
                                    c->stream));
        k_rescue_lattice_points<<<grid1d(nl), 256, 0, c->stream>>>(
            g, gl, cand, ncand, c->gr_rl_idx.as<int64_t>(), c->gr_rl_xy.as<float2>());
        COUNT_LAUNCH(c);
        TRY(bbkde::surrogate_infer(sur, c->stream, nl, c->gr_rl_xy.as<float2>(), 0, 0.0, 0.0,
                                   0.0, 0.0, c->gr_rl_net.as<float>()) == BBKDE_OK
                ? BBKDE_OK
                : fail(c, BBKDE_CUDA_ERROR, "grid: surrogate inference failed"));
        COUNT_LAUNCH(c);
        k_scatter_net<<<grid1d(nl), 256, 0, c->stream>>>(
            c->gr_rl_idx.as<int64_t>(), c->gr_rl_net.as<float>(), nl, c->gr_lat_net.as<float>());
        COUNT_LAUNCH(c);
        lat_net = c->gr_lat_net.as<float>();
        if (P == 9) {
          TRY(quarter_net());
          q_net = c->gr_q_net.as<float>();
        }
        k_anchor_residual<<<grid1d(n_anchor), 256, 0, c->stream>>>(
            c->gr_lat_exact.as<double>(), lat_net, g.ntx, g.nty, c->gr_resid.as<float>());
        COUNT_LAUNCH(c);
        const int64_t np = (int64_t)ncand * T * T;
        TRY(ensure(c, c->gr_cand_xy, (size_t)np * sizeof(float2)));
        TRY(ensure(c, c->gr_cand_net, (size_t)np * sizeof(float)));
        k_tile_points<<<grid1d(np), 256, 0, c->stream>>>(g, cand, np,
                                                        c->gr_cand_xy.as<float2>());
        COUNT_LAUNCH(c);
        TRY(bbkde::surrogate_infer(sur, c->stream, np, c->gr_cand_xy.as<float2>(), 0, 0.0, 0.0,
                                   0.0, 0.0, c->gr_cand_net.as<float>()) == BBKDE_OK
                ? BBKDE_OK
                : fail(c, BBKDE_CUDA_ERROR, "grid: surrogate inference failed"));
        COUNT_LAUNCH(c);
        k_tile_predict_list<<<(unsigned)ncand, 256, 0, c->stream>>>(
            g, cand, c->gr_cand_net.as<float>(), resid, interp, pred, c->gr_bad.as<int>());
        COUNT_LAUNCH(c);
        pa.list = cand;
        pa.n_list = ncand;
        pa.lat_net = lat_net;
        pa.q_net = q_net;
        k_probe_check<<<grid1d(ncand), 256, 0, c->stream>>>(pa);
        COUNT_LAUNCH(c);
        k_rescue_update<<<grid1d(ncand), 256, 0, c->stream>>>(
            cand, ncand, c->gr_bad.as<int>(), c->gr_terr.as<unsigned>(), (float)cfg->rel_tol,
            c->gr_flag.as<int>());
        COUNT_LAUNCH(c);
        CUDA_TRY(c, cudaMemsetAsync(c->gr_counts.as<unsigned long long>() + 1, 0,
                                    2 * sizeof(unsigned long long), c->stream));
        k_flag_recount<<<grid1d(ntiles), 256, 0, c->stream>>>(fa);
        COUNT_LAUNCH(c);
        CUDA_TRY(c, cudaGetLastError());
      }
      CUDA_TRY(c, cudaEventRecord(c->ev2, c->stream));
    }
    // 6. Predicted values on the tiles that keep them.
    const dim3 ab((unsigned)std::min<int64_t>((g.nx + 1023) / 1024, 16),
                  (unsigned)std::min<int64_t>(g.ny, (int64_t)c->sm_count * 8));
    k_apply<<<ab, 256, 0, c->stream>>>(g, T == 32 ? 5 : 4, c->gr_pred.as<float>(),
                                       c->gr_flag.as<int>(), out);
    COUNT_LAUNCH(c);
  }
  // 7. Exact fallback on the flagged tiles.
  CUDA_TRY(c, cudaGetLastError());
  size_t tmp = 0;
  CUDA_TRY(c, cub::DeviceSelect::Flagged(nullptr, tmp, c->gr_order.as<int>(),
                                         c->gr_flag_ord.as<int>(), c->gr_list.as<int>(),
                                         c->gr_nsel.as<int>(), (int)ntiles, c->stream));
  TRY(ensure(c, c->ms_tmp, tmp));
  CUDA_TRY(c, cub::DeviceSelect::Flagged(c->ms_tmp.p, tmp, c->gr_order.as<int>(),
                                         c->gr_flag_ord.as<int>(), c->gr_list.as<int>(),
                                         c->gr_nsel.as<int>(), (int)ntiles, c->stream));
  c->launch_total += 2;
  int nsel = 0;
  unsigned long long counts[3] = {0, 0, 0};
  CUDA_TRY(c, cudaMemcpyAsync(&nsel, c->gr_nsel.p, sizeof(int), cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaMemcpyAsync(counts, c->gr_counts.p, sizeof(counts), cudaMemcpyDeviceToHost,
                              c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  TRY(grid_exact(c, r, g, c->gr_list.as<int>(), nsel, cfg->cull_rel, full, out, &st.pairs,
                 &st.max_bound_ratio, cfg->pair_form != 0, cfg->tensor_cores));
  CUDA_TRY(c, cudaEventRecord(c->ev3, c->stream));
  // Points in the flagged tiles (edge tiles may be partial).
  std::vector<int> flags((size_t)ntiles);
  CUDA_TRY(c, cudaMemcpyAsync(flags.data(), c->gr_flag.p, (size_t)ntiles * sizeof(int),
                              cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  int64_t fb_points = 0;
  for (int64_t t = 0; t < ntiles; ++t) {
    if (!flags[(size_t)t]) continue;
    const int64_t tx = t % g.ntx, ty = t / g.ntx;
    fb_points += std::min<int64_t>(T, g.nx - tx * T) * std::min<int64_t>(T, g.ny - ty * T);
  }
  float ms = 0.f;
  CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev3));
  st.ms_total = ms;
  float ms01 = 0.f, ms12 = 0.f;
  CUDA_TRY(c, cudaEventElapsedTime(&ms01, c->ev0, c->ev1));
  CUDA_TRY(c, cudaEventElapsedTime(&ms12, c->ev1, c->ev2));
  st.ms_predict = rescue ? ms12 : ms01;
  st.ms_probe = rescue ? ms01 : ms12;
  CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev2, c->ev3));
  st.ms_fallback = ms;
  st.tiles_low = (int64_t)counts[0];
  st.tiles_flagged = (int64_t)counts[1];
  st.tiles_surrogate = ntiles - st.tiles_flagged;
  st.exact_points += fb_points;
  unsigned eb = (unsigned)counts[2];
  float pe = 0.f;
  std::memcpy(&pe, &eb, sizeof(pe));
  st.max_probe_err = mode == BBKDE_GRID_EXACT ? 0.0 : (double)pe;
  c->last_ms = st.ms_total;
  c->last_pairs = st.pairs;
  c->last_launches = 0;
  if (stats) *stats = st;
  if (mode != BBKDE_GRID_EXACT && sur && bbkde::surrogate_check(sur) != BBKDE_OK)
    return fail(c, BBKDE_TIMEOUT, "grid: surrogate inference wait expired");
  return BBKDE_OK;
}

// Least-squares CV with numerical integration (KernelDensityImpl.h:14-97): the
// square integral is the culled exact density on the grid (bound 1e-7) summed
// as f^2 dx dy in FP64; the leave-one-out term is the weighted self-sum with the
// diagonal excluded (the reference subtracts the self term, :50-60).
extern "C" int bbkde_lsq_numint_cv(bbkde_ctx *c, const bbkde_kernel_desc *k,
                                   const bbkde_grid *grid, int precision, double *cv_out) {
  Resolved r;
  TRY(self_checks(c, k, precision, r));
  if (!cv_out || !grid) return fail(c, BBKDE_INVALID_ARGUMENT, "NULL argument");
  if (precision != BBKDE_FP32C)
    return fail(c, BBKDE_UNSUPPORTED,
                "lsq_numint_cv: FP32C only (the grid term is the culled FP32 sum)");
  if (r.dim != 2) return fail(c, BBKDE_INVALID_ARGUMENT, "lsq_numint_cv: 2-D kernels only");
  TRY(culled_kernel_ok(c, r));
  PointSet &s = c->sets[BBKDE_REFERENCE];
  if (s.n == 0) { *cv_out = 0.0; return BBKDE_OK; }
  if (grid->nx < 1 || grid->ny < 1)
    return fail(c, BBKDE_INVALID_ARGUMENT, "grid: need nx, ny >= 1");
  // Leave-one-out term (:40-60).
  TRY(ensure(c, c->out_dev, (size_t)s.n * sizeof(double)));
  TRY(pair_sum(c, r, precision, BBKDE_REFERENCE, 0, s.n - 1, 0, s.n - 1, r.norm, true,
               c->out_dev.as<double>(), EPI_W_VALUE, s.weight.as<double>()));
  double llo = 0.0;
  CUDA_TRY(c, cudaMemcpy(&llo, c->scalars.p, sizeof(double), cudaMemcpyDeviceToHost));
  const double ms_loo = c->last_ms, pairs_loo = c->last_pairs;
  // Square integral over the grid (:62-93).
  const int64_t npts = grid->nx * grid->ny;
  TRY(ensure(c, c->gr_out, (size_t)npts * sizeof(double)));
  bbkde_grid_config cfg = {BBKDE_GRID_EXACT, 16, 1, 1, 1e-3, 0.0, 1e-7, 1, 0, 0};
  bbkde_grid_stats st;
  TRY(bbkde_eval_grid(c, nullptr, k, grid, &cfg, c->gr_out.as<double>(), &st));
  const unsigned nb = std::min<unsigned>(grid1d(npts, kRedBlock), 4096u);
  TRY(ensure(c, c->block_sums, (size_t)nb * sizeof(double)));
  k_sum_sq<<<nb, kRedBlock, 0, c->stream>>>(c->gr_out.as<double>(), npts,
                                            c->block_sums.as<double>());
  COUNT_LAUNCH(c);
  k_sum_blocks<<<1, kRedBlock, 0, c->stream>>>(c->block_sums.as<double>(), nb,
                                               c->scalars.as<double>() + 2);
  COUNT_LAUNCH(c);
  CUDA_TRY(c, cudaGetLastError());
  double sum_sq = 0.0;
  CUDA_TRY(c, cudaMemcpyAsync(&sum_sq, c->scalars.as<double>() + 2, sizeof(double),
                              cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const double dx = (grid->x1 - grid->x0) / grid->nx, dy = (grid->y1 - grid->y0) / grid->ny;
  *cv_out = sum_sq * dx * dy - 2 * llo;   // :95
  c->last_ms = ms_loo + st.ms_total;
  c->last_pairs = pairs_loo + st.pairs;
  c->last_launches = 0;
  return BBKDE_OK;
}

// ===========================================================================
// Allocation-free direct evaluation (bbkde_eval_noalloc)
//
// For callers that must not allocate device memory: code that runs inside a
// host framework owning every device allocation through its own pool (so a
// cudaMalloc from a library would fragment or bypass it), work enqueued while
// the process has memory-allocation checks that forbid new allocations, or
// code paths that have to run when device memory is exhausted. Such callers
// pass device pointers for every input and output; the scratch the pair sum
// needs (packed reference records, FP32 query coordinates and the FP64 segment
// partials) lives in one fixed array of the library's device image.
// ===========================================================================

// 64 MiB of device scratch. Every device that loads libbbkde.so holds it until
// the process exits. Host code must not use this name as an address: on the
// host it is only a stand-in for the device symbol, which is why the entry point
// resolves its device address with cudaGetSymbolAddress.
static constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

void noalloc_msg(char *buf, int64_t len, const char *fmt, ...) {
  if (!buf || len <= 0) return;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, (size_t)len, fmt, ap);
  va_end(ap);
}

inline size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Device address of g_noalloc_scratch in the current context. Resolved on every
// call (a lookup once the module is loaded), so a device reset or a different
// current context never leaves a stale pointer behind. The first resolution on a
// device loads the library's module there (CUDA loads modules lazily), which
// places the array in that device's memory.
int noalloc_scratch(void **out, char *err, int64_t errlen) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    noalloc_msg(err, errlen, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    cudaGetLastError();
    return BBKDE_CUDA_ERROR;
  }
  *out = p;
  return BBKDE_OK;
}

}  // namespace

extern "C" int bbkde_eval_noalloc(const bbkde_kernel_desc *kernel, int64_t n_ref,
                                  const double *ref_x, const double *ref_y,
                                  const double *ref_mass, const double *ref_abw,
                                  int64_t n_query, const double *query_x,
                                  const double *query_y, int normalized, double *out,
                                  void *stream, char *errbuf, int64_t errbuf_len) {
  if (errbuf && errbuf_len > 0) errbuf[0] = '\0';
  Resolved r;
  if (resolve(nullptr, kernel, r) != BBKDE_OK) {
    noalloc_msg(errbuf, errbuf_len, "invalid kernel descriptor (kind, dim or bandwidths)");
    return BBKDE_INVALID_ARGUMENT;
  }
  const int dim = r.dim;
  if (n_ref < 1 || n_query < 0) {
    noalloc_msg(errbuf, errbuf_len, "need n_ref >= 1 and n_query >= 0");
    return BBKDE_INVALID_ARGUMENT;
  }
  // Resolve the scratch before anything else, so that a call with no queries loads
  // the array on this device (a cheap warm-up before capture or memory pressure).
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) {
    noalloc_msg(errbuf, errbuf_len, "cudaGetDevice: %s", cudaGetErrorString(e));
    return BBKDE_CUDA_ERROR;
  }
  void *base = nullptr;
  int rc = noalloc_scratch(&base, errbuf, errbuf_len);
  if (rc != BBKDE_OK) return rc;
  if (n_query == 0) return BBKDE_OK;
  if (!ref_x || !ref_mass || !query_x || !out || (dim == 2 && (!ref_y || !query_y))) {
    noalloc_msg(errbuf, errbuf_len, "a required device pointer is NULL");
    return BBKDE_INVALID_ARGUMENT;
  }
  // Bound the counts before any byte arithmetic, so that no product can wrap.
  if (n_ref > (int64_t)(kNoAllocScratchBytes / 16) ||
      n_query > (int64_t)(kNoAllocScratchBytes / 12)) {
    noalloc_msg(errbuf, errbuf_len,
                "n_ref = %lld or n_query = %lld exceeds the %zu bytes of scratch of the "
                "allocation-free entry point; use bbkde_eval_range for larger problems",
                (long long)n_ref, (long long)n_query, kNoAllocScratchBytes);
    return BBKDE_OUT_OF_RANGE;
  }
  // Scratch layout: records | extra column | query x | query y | partials.
  const bool ext = op_has_extra(r.op);
  const size_t off_ext = align256((size_t)n_ref * sizeof(float4));
  const size_t off_qx = off_ext + (ext ? align256((size_t)n_ref * sizeof(float)) : 0);
  const size_t off_qy = off_qx + align256((size_t)n_query * sizeof(float));
  const size_t off_part = off_qy + (dim == 2 ? align256((size_t)n_query * sizeof(float)) : 0);
  const size_t per_seg = (size_t)n_query * sizeof(double);
  if (off_part + per_seg > kNoAllocScratchBytes) {
    noalloc_msg(errbuf, errbuf_len,
                "n_ref = %lld and n_query = %lld need %zu bytes of scratch, more than the "
                "%zu bytes of the allocation-free entry point (16-20 B per reference, "
                "4 B per query coordinate, 8 B per query and reference segment); use "
                "bbkde_eval_range for larger problems",
                (long long)n_ref, (long long)n_query, off_part + per_seg,
                kNoAllocScratchBytes);
    return BBKDE_OUT_OF_RANGE;
  }
  unsigned char *sb = static_cast<unsigned char *>(base);
  float4 *rec = reinterpret_cast<float4 *>(sb);
  float *extc = ext ? reinterpret_cast<float *>(sb + off_ext) : nullptr;
  float *qx = reinterpret_cast<float *>(sb + off_qx);
  float *qy = dim == 2 ? reinterpret_cast<float *>(sb + off_qy) : qx;
  double *partial = reinterpret_cast<double *>(sb + off_part);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  PackArgs p;
  p.x = ref_x;
  p.y = ref_y;
  p.mass = ref_mass;
  p.abw = ref_abw;
  p.n = n_ref;
  p.op = r.op;
  p.dim = dim;
  p.c1 = r.c1_f32;
  p.c2 = r.c2_f32;
  p.h1 = r.h1;
  p.h2 = r.h2;
  p.mass_scale = r.mass_scale;
  k_pack_f32<<<grid1d(n_ref), 256, 0, st>>>(p, rec, extc);
  k_to_f32<<<grid1d(n_query), 256, 0, st>>>(query_x, qx, n_query);
  if (dim == 2) k_to_f32<<<grid1d(n_query), 256, 0, st>>>(query_y, qy, n_query);

  // Segment the reference range as the context path does, within the scratch.
  int sm_count = 0;
  e = cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess || sm_count < 1) {
    noalloc_msg(errbuf, errbuf_len, "cudaDeviceGetAttribute(SM count): %s",
                cudaGetErrorString(e));
    cudaGetLastError();
    return BBKDE_CUDA_ERROR;
  }
  const int variant = kDefaultVariant;
  const int qpb = queries_per_block(variant, false);
  const int64_t qtiles = (n_query + qpb - 1) / qpb;
  const int64_t target = (int64_t)sm_count * 4 * 16;
  int64_t nseg = std::max<int64_t>(1, (target + qtiles - 1) / qtiles);
  nseg = std::min<int64_t>(nseg, std::max<int64_t>(1, (n_ref + 511) / 512));
  nseg = std::min<int64_t>(nseg, (int64_t)((kNoAllocScratchBytes - off_part) / per_seg));
  nseg = std::min<int64_t>(nseg, 65535);
  int64_t seg_len = (n_ref + nseg - 1) / nseg;
  seg_len = (seg_len + kTile - 1) / kTile * kTile;
  nseg = std::max<int64_t>(1, (n_ref + seg_len - 1) / seg_len);

  SumArgs a;
  a.refs = rec;
  a.extra = extc;
  a.qx = qx;
  a.qy = qy;
  a.r_begin = 0;
  a.r_end = n_ref;
  a.seg_len = seg_len;
  a.q_begin = 0;
  a.q_count = n_query;
  a.exclude_self = 0;
  a.scale = 1.0;
  a.out = partial;   // every (segment, query) entry is written: nothing to clear
  a.status = nullptr;
  dim3 grid((unsigned)qtiles, (unsigned)nseg);
  if (dim == 2) dispatch_op<2>(r.op, false, variant, grid, st, a);
  else dispatch_op<1>(r.op, false, variant, grid, st, a);
  k_combine<<<grid1d(n_query, kRedBlock), kRedBlock, 0, st>>>(
      partial, (int)nseg, n_query, normalized ? r.norm : 1.0, out, EPI_NONE, nullptr, nullptr);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    noalloc_msg(errbuf, errbuf_len, "kernel launch: %s", cudaGetErrorString(e));
    return BBKDE_CUDA_ERROR;
  }
  return BBKDE_OK;
}
