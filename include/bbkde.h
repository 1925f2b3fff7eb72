/* bbkde.h -- C ABI of the B200 direct kernel-density library (libbbkde.so).
 *
 * This is the drop-in boundary for bbrcit_kde's direct N-body density path. Every
 * entry point below replaces one piece of the reference's CudaDirectKde<> /
 * KernelDensity<> path (file:line cited per function; paths are relative to the
 * reference project root). Signatures use plain pointers and sizes only.
 *
 * Conventions
 *   - Every call returns an int status (bbkde_status). BBKDE_OK is 0. On failure
 *     bbkde_ctx_last_error() holds a message.
 *   - Calls are synchronous from the caller's point of view: when a call returns,
 *     host outputs are written and device work for the call has finished.
 *   - Host arrays are caller-owned; the library copies what it needs.
 *   - Coordinates are AoS with stride `dim` (x0,y0,x1,y1,... for dim 2).
 *   - Index ranges are closed intervals [i, j], as in the reference.
 *   - One context per host thread; distinct contexts may be used concurrently.
 */
#ifndef BBKDE_H_
#define BBKDE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BBKDE_ABI_VERSION 2

#if defined(__GNUC__)
#define BBKDE_API __attribute__((visibility("default")))
#else
#define BBKDE_API
#endif

typedef struct bbkde_ctx bbkde_ctx;

/* Status codes. The C++ wrapper (include/bbkde/) maps OUT_OF_RANGE to
 * std::out_of_range and INVALID_ARGUMENT to std::invalid_argument, as the
 * reference throws them (CudaDirectKde.h:181-190, KernelDensityImpl.h:301-303). */
typedef enum {
  BBKDE_OK = 0,
  BBKDE_OUT_OF_RANGE = 1,
  BBKDE_INVALID_ARGUMENT = 2,
  BBKDE_CUDA_ERROR = 3,
  BBKDE_TIMEOUT = 4,
  BBKDE_UNSUPPORTED = 5,
  BBKDE_NO_DEVICE = 6,
  BBKDE_ALLOC_FAILED = 7
} bbkde_status;

/* Kernel families (the include/Kernels/ headers of the reference). */
typedef enum {
  BBKDE_GAUSSIAN = 0,                   /* GaussianKernel<D,T>, D = 1, 2 */
  BBKDE_EPANECHNIKOV = 1,               /* EpanechnikovKernel<D,T>, D = 1, 2 */
  BBKDE_GAUSSIAN_PRODUCT_2D = 2,        /* GaussianProductKernel2d<T> */
  BBKDE_EPANECHNIKOV_PRODUCT_2D = 3,    /* EpanechnikovProductKernel2d<T> */
  BBKDE_GAUSSIAN_PRODUCT_CONV_2D = 4,   /* GaussianProductConvKernel2d<T> */
  BBKDE_EPANECHNIKOV_PRODUCT_CONV_2D = 5,/* EpanechnikovProductConvKernel2d<T> */
  BBKDE_GAUSSIAN_CONV_1D = 6,           /* GaussianConvKernel1d<T> */
  BBKDE_EPANECHNIKOV_CONV_1D = 7        /* EpanechnikovConvKernel1d<T> */
} bbkde_kernel_kind;

/* Arithmetic of the pair sum.
 *   FP32C: FP32 kernel evaluation (MUFU ex2 for the Gaussians), Kahan-compensated
 *          FP32 partial sums, FP64 cross-block combination and normalisation.
 *   FP64 : FP64 throughout (the reference's CPU arithmetic). */
typedef enum { BBKDE_FP32C = 0, BBKDE_FP64 = 1 } bbkde_precision;

/* Which point set an upload fills: the reference points of CudaDirectKde<>
 * (ref_pts) or its query points (query_pts), CudaDirectKde.h:57-59. */
typedef enum { BBKDE_REFERENCE = 0, BBKDE_QUERY = 1 } bbkde_role;

/* Kernel descriptor flags. */
enum {
  /* GaussianProductConvKernel2d: the reference's float/double specialisations
   * evaluate exp(-0.5 arg) (KernelTraits.h:431-433, :444-446) although the
   * convolution of two Gaussians is exp(-0.25 arg) (KernelTraits.h:418-420).
   * By default the library reproduces the reference; this flag selects -0.25. */
  BBKDE_FLAG_EXACT_GAUSS_CONV = 1
};

typedef struct {
  int32_t kind;      /* bbkde_kernel_kind */
  int32_t dim;       /* 1 or 2 */
  double h[2];       /* bandwidth (h[0]) or (hx, hy) for the 2-D product kernels */
  int32_t flags;     /* BBKDE_FLAG_* */
  int32_t reserved;  /* must be 0 */
} bbkde_kernel_desc;

/* ---- library / context ------------------------------------------------- */

BBKDE_API int bbkde_abi_version(void);
BBKDE_API const char *bbkde_status_string(int status);

/* Create a context on CUDA device `device`. The context owns its device buffers
 * and a non-blocking stream. Replaces the implicit device state of
 * CudaDirectKde<> (CudaDirectKde.h:109-116). */
BBKDE_API int bbkde_ctx_create(int device, bbkde_ctx **out);
BBKDE_API int bbkde_ctx_destroy(bbkde_ctx *ctx);
BBKDE_API const char *bbkde_ctx_last_error(const bbkde_ctx *ctx);

/* Run the context's work on `stream` (a cudaStream_t), or on its own stream
 * when `stream` is NULL. */
BBKDE_API int bbkde_ctx_set_stream(bbkde_ctx *ctx, void *stream);

/* ---- point sets ---------------------------------------------------------- */

/* Upload n points of dimension dim into the REFERENCE or QUERY set, replacing it.
 * Replaces CudaDirectKde(ref_pts, query_pts) / alloc_copy_host_dev_points
 * (CudaDirectKde.h:330-374), which copies {x, y, mass, abw} per point
 * (Point2d.h:31-38). Any of mass / abw / weight may be NULL: mass defaults to 1,
 * abw to 1, weight to mass. Weights are only used by bbkde_adapt_density and the
 * cross-validation calls (the `weight` attribute, AdaKdeAttributes.h:36-37).
 * n == 0 empties the set. */
BBKDE_API int bbkde_upload(bbkde_ctx *ctx, int role, int dim, int64_t n, const double *coords,
                 const double *mass, const double *abw, const double *weight);

/* Number of points in a set (CudaDirectKde::reference_size / query_size,
 * CudaDirectKde.h:290-297). Returns -1 on a bad context or role. */
BBKDE_API int64_t bbkde_size(const bbkde_ctx *ctx, int role);

/* Copy the REFERENCE set's current mass and abw back to the host (either may be
 * NULL). After bbkde_adapt_density these are the adapted values. */
BBKDE_API int bbkde_download_attributes(bbkde_ctx *ctx, double *mass, double *abw);

/* ---- direct evaluation --------------------------------------------------- */

/* For every query k in [q_i, q_j]:
 *   out[k - q_i] = [C(h) *] sum_{r in [r_i, r_j]} mass_r * U(q_k, x_r; h * abw_r)
 * Replaces CudaDirectKde::eval (normalized = 1) and unnormalized_eval
 * (normalized = 0), CudaDirectKde.h:176-229, and the eval_kernel launch inside it
 * (:126-173). Closed ranges; j >= size gives OUT_OF_RANGE and i > j gives
 * INVALID_ARGUMENT, as the reference's checks (:181-190). `out` is host memory
 * of length q_j - q_i + 1. `block_size` is accepted as a tuning hint, as in the
 * reference (0 = automatic). */
BBKDE_API int bbkde_eval_range(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel, int64_t r_i,
                     int64_t r_j, int64_t q_i, int64_t q_j, int normalized,
                     int precision, double *out, int64_t block_size);

/* As bbkde_eval_range, but `out_device` is device memory on the context's device
 * (for callers that keep results on the GPU). */
BBKDE_API int bbkde_eval_range_device(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel,
                            int64_t r_i, int64_t r_j, int64_t q_i, int64_t q_j,
                            int normalized, int precision, double *out_device,
                            int64_t block_size);

/* ---- adaptive densities (Silverman 5.3) ---------------------------------- */

/* KernelDensity::adapt_density(alpha) (KernelDensityImpl.h:291-359) over the
 * REFERENCE set with exact direct sums: pilot_i = C sum_j w_j U(x_i, x_j; h)
 * (self term included, abw = 1), g = exp(sum_i w_i log pilot_i),
 * abw_i = (pilot_i / g)^-alpha, mass_i = w_i abw_i^-dim. The adapted abw and
 * mass replace the set's attributes on the device. Weights are used as given
 * (KernelDensity normalises them to sum 1 before this call). alpha outside
 * [0, 1] returns INVALID_ARGUMENT; alpha == 0 resets abw = 1, mass = w.
 * Any output pointer may be NULL (host memory, length n, or one double for g). */
BBKDE_API int bbkde_adapt_density(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel, double alpha,
                        int precision, double *abw_out, double *mass_out,
                        double *pilot_out, double *g_out);

/* As bbkde_adapt_density, with the pilot to a tolerance, as the reference's
 * adapt_density(alpha, rel_err, abs_err) evaluates it through its tree
 * (KernelDensityImpl.h:291-359): the culled self-sum (see bbkde_eval_tol),
 * every pilot value f within max(rel_tol f, abs_tol) / 2 of the full sum plus
 * the FP32-compensated arithmetic error (0 <= rel_tol < 1, abs_tol >= 0 in
 * density units; both 0 sum every pair that does not flush to zero in FP32);
 * g and the attributes in FP64 as above. The Epanechnikov convolution kernels
 * give UNSUPPORTED. */
BBKDE_API int bbkde_adapt_density_tol(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel,
                                      double alpha, double rel_tol, double abs_tol,
                                      double *abw_out, double *mass_out, double *pilot_out,
                                      double *g_out);

/* KernelDensity::unadapt_density (KernelDensityImpl.h:254-273): abw = 1, mass = w. */
BBKDE_API int bbkde_unadapt_density(bbkde_ctx *ctx);

/* ---- cross-validation ---------------------------------------------------- */

/* KernelDensity::likelihood_cross_validate (KernelDensityImpl.h:215-252) with
 * exact sums over the REFERENCE set: sum_i w_i log(f_i), where f_i is the
 * leave-one-out density C sum_{j != i} m_j U(x_i, x_j; h abw_j). The diagonal is
 * excluded rather than subtracted; see the design notes. */
BBKDE_API int bbkde_likelihood_cv(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel, int precision,
                        double *cv_out);

/* KernelDensity::lsq_convolution_cross_validate (KernelDensityImpl.h:142-209):
 * sum_i w_i fconv_i - 2 sum_i w_i f_i, fconv the all-pairs sum with the
 * kernel's convolution kernel (ConvKernelAssociator.h). Defined for GAUSSIAN
 * and EPANECHNIKOV with dim 1, and for the two 2-D product kernels. */
BBKDE_API int bbkde_lsq_conv_cv(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel, int precision,
                      double *cv_out);

/* Cross validation with the density sums to a tolerance, as the reference
 * evaluates them through its tree (likelihood_cross_validate(rel_err, abs_err),
 * KernelDensityImpl.h:215-252; lsq_convolution_cross_validate, :142-209): every
 * full self-sum f is a culled sum within max(rel_tol f, abs_tol) / 2 of the exact
 * one (0 <= rel_tol < 1, abs_tol >= 0; FP32-compensated), and the leave-one-out
 * value is that sum minus the self term
 * m_i C(h), as the reference computes it (its FP32 mass, so the subtraction
 * cancels the self term of the sum). FP64 totals in fixed order. Kernels whose
 * culled sum is unsupported (the Epanechnikov convolution kernels, hence the
 * Epanechnikov product LSQ) give UNSUPPORTED. */
BBKDE_API int bbkde_likelihood_cv_tol(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel,
                                      double rel_tol, double abs_tol, double *cv_out);
BBKDE_API int bbkde_lsq_conv_cv_tol(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel,
                                    double rel_tol, double abs_tol, double *cv_out);

/* ---- batched cross-validation -------------------------------------------- */

typedef struct {
  int64_t n;              /* points in this dataset */
  const double *coords;   /* host, AoS (x0, y0, x1, y1, ...) */
  const double *weights;  /* host, n raw weights (normalised to sum 1 here); NULL = 1 */
} bbkde_dataset;

/* Likelihood and least-squares (convolution) cross-validation of many 2-D
 * datasets over a bandwidth grid hx[0..n_hx) x hy[0..n_hy) in one call:
 *   lik_out[(s * n_hx + a) * n_hy + b] = likelihood_cross_validate of dataset s
 *       with the product kernel (hx[a], hy[b])   (KernelDensityImpl.h:215-252)
 *   lsq_out[...]                       = lsq_convolution_cross_validate
 *                                                (KernelDensityImpl.h:142-209)
 * which the reference computes one bandwidth at a time in a host loop
 * (grid_search/grid_search.cc:370-402). Weights are normalised per dataset and
 * masses equal weights (non-adaptive), leave-one-out excludes the diagonal.
 *   BBKDE_EPANECHNIKOV_PRODUCT_2D: one persistent launch for every dataset and
 *     bandwidth (moment binning, FP64), captured in a CUDA graph and replayed
 *     for repeated calls of the same shape.
 *   BBKDE_GAUSSIAN_PRODUCT_2D: exact per-bandwidth loop over the pair sum.
 * hx and hy must be strictly increasing, positive, at most 64 values each.
 * Exact-duplicate points are not merged (the reference's Kd-tree merges them). */
BBKDE_API int bbkde_cv_batch(bbkde_ctx *ctx, int kind, int n_sets, const bbkde_dataset *sets,
                             int n_hx, const double *hx, int n_hy, const double *hy,
                             int precision, double *lik_out, double *lsq_out);

/* Statistics of the last bbkde_cv_batch launch on this context: the in-support
 * pair counts (the units of its shared-memory bound) -- lik_pairs ordered pairs
 * with |dx| < hx_max and |dy| < hy_max (4 64-bit shared-memory atomic adds each),
 * conv_pairs unordered pairs with |dx| < 2 hx_max and |dy| < 2 hy_max (16 each)
 * -- and the work-item plan it ran, of n_plans. Any pointer may be NULL. No
 * reference counterpart. */
BBKDE_API int bbkde_cv_batch_info(const bbkde_ctx *ctx, int64_t *lik_pairs, int64_t *conv_pairs,
                                  int *plan, int *n_plans);

/* Work-item plan of the batched CV launch (likelihood items of 4096, 1024 or 2048
 * queries; convolution items of up to 256, 256 or 128 queries of one grid cell).
 * By default (-1) the context autotunes per problem class (number of sets, log2
 * of the total points and of the pair count, grid shape): the first calls of a
 * class each run a plan not yet tried -- every call returns complete results --
 * and later calls keep the fastest measured. Results of different plans agree
 * to FP64 rounding (the likelihood sums are grouped by item). plan in
 * [0, n_plans) forces that plan. No reference counterpart. */
BBKDE_API int bbkde_ctx_set_cv_plan(bbkde_ctx *ctx, int plan);

/* ---- learned log-density surrogate ---------------------------------------- */

/* A small network (2 -> 128 -> 128 -> 128 -> 1, SiLU) for log-density, trained
 * with hand-written BF16 tensor-core forward / backward kernels (FP32 accumulate)
 * on exact densities computed by the pair sums, and evaluated with a fused BF16
 * tensor-core inference kernel. No reference counterpart: the reference evaluates
 * every query with a density sum (KernelDensityImpl.h:1157-1231); the surrogate
 * stands in for that sum on dense query grids, with the exact sum as its fallback
 * and judge (bbkde_eval_grid). */
typedef struct bbkde_surrogate bbkde_surrogate;

typedef struct {
  int64_t steps;     /* optimiser steps */
  int64_t batch;     /* points per step (>= 64) */
  double lr;         /* initial learning rate (Adam) */
  double lr_final;   /* learning rate at the last step (cosine decay) */
  double beta1, beta2, eps;   /* Adam; 0 selects 0.9, 0.999, 1e-8 */
  uint64_t seed;     /* mini-batch sampling seed */
} bbkde_train_config;

/* Create a surrogate on `device` with seeded Glorot-uniform weights. */
BBKDE_API int bbkde_surrogate_create(int device, uint64_t seed, bbkde_surrogate **out);
BBKDE_API int bbkde_surrogate_destroy(bbkde_surrogate *s);
BBKDE_API const char *bbkde_surrogate_last_error(const bbkde_surrogate *s);

/* Number of FP32 parameters: W1[128][2] b1[128] W2[128][128] b2[128]
 * W3[128][128] b3[128] w4[128] b4. norm6 = {cx, cy, sx, sy, mu, sigma}: the
 * network sees ((x - cx) sx, (y - cy) sy) and predicts (log f - mu) / sigma. */
BBKDE_API int bbkde_surrogate_num_params(void);
BBKDE_API int bbkde_surrogate_set_params(bbkde_surrogate *s, const float *params,
                                         const float *norm6);
BBKDE_API int bbkde_surrogate_get_params(bbkde_surrogate *s, float *params, float *norm6);

/* Gradient of the mean squared error in normalised units over all n points
 * (host xy AoS, host log-density targets), one forward + backward pass on the
 * tensor cores without an update; grad has bbkde_surrogate_num_params() floats. */
BBKDE_API int bbkde_surrogate_gradient(bbkde_surrogate *s, int64_t n, const double *xy,
                                       const double *target, float *grad, double *loss);

/* Train on n (xy, log-density) rows; sets the input / output normalisation from
 * the data. final_loss = the last step's mini-batch loss (normalised units). */
BBKDE_API int bbkde_surrogate_train(bbkde_surrogate *s, int64_t n, const double *xy,
                                    const double *target, const bbkde_train_config *cfg,
                                    double *final_loss);

/* Predicted log-density: host arrays, synchronous. */
BBKDE_API int bbkde_surrogate_predict(bbkde_surrogate *s, int64_t n, const double *xy,
                                      double *out);
/* Device float2 points -> device floats, asynchronous on the surrogate's stream. */
BBKDE_API int bbkde_surrogate_predict_device(bbkde_surrogate *s, int64_t n, const void *xy_f2,
                                             float *out);

/* Inference precision: 0 (default) = BF16 activations, as in training;
 * 1 = two-term BF16 activations (a = hi + lo, both BF16, same BF16 weights, FP32
 * accumulate): relative activation rounding ~2^-17 instead of ~2^-9 at twice the
 * tensor-core work. */
BBKDE_API int bbkde_surrogate_set_inference(bbkde_surrogate *s, int split_activations);

/* Tensor-core engine of inference, training and bbkde_surrogate_gradient:
 * BBKDE_ENGINE_TCGEN05 (default; tcgen05.mma with TMEM accumulators, 128-point
 * tiles; the backward products read the stored BF16 matrices transposed as
 * MN-major operands) or BBKDE_ENGINE_MMA_SYNC (mma.sync.m16n8k16, 16 points per
 * warp). Inference: same arithmetic, results agree to FP32 summation order.
 * Training: the tcgen05 step keeps pre-activations and input gradients in FP32
 * (TMEM) and rounds to BF16 only the operands of the products; the mma.sync step
 * also stores pre-activations and gradients as BF16. */
enum { BBKDE_ENGINE_TCGEN05 = 0, BBKDE_ENGINE_MMA_SYNC = 1 };
BBKDE_API int bbkde_surrogate_set_engine(bbkde_surrogate *s, int engine);

/* Checkpoint: magic "BBKDEMLP", version, parameter count, normalisation, FP32
 * parameters (little-endian). */
BBKDE_API int bbkde_surrogate_save(bbkde_surrogate *s, const char *path);
BBKDE_API int bbkde_surrogate_load(bbkde_surrogate *s, const char *path);

/* ---- culled direct evaluation and dense grids ------------------------------ */

/* Culled direct evaluation: the QUERY set against every REFERENCE point, summing
 * only the reference tiles (256 Morton-ordered points) that can contribute. For
 * the Gaussian kernels the part left out is bounded, per block of queries, by
 * rel_tol times the smallest sum in that block, so every result is within
 * rel_tol (plus the FP32-compensated arithmetic error) of the full sum; for the
 * Epanechnikov kernels only tiles entirely outside the support are skipped
 * (exact). Kernels: Gaussian (1-D, 2-D), Epanechnikov (1-D, 2-D), the 2-D
 * product kernels and the Gaussian convolution kernels; the Epanechnikov
 * convolution kernels are BBKDE_UNSUPPORTED. No reference counterpart in this
 * form: it plays the part of the reference's tree-pruned evaluation
 * (KernelDensityImpl.h:548-640) with a deterministic error bound. out holds
 * bbkde_size(QUERY) doubles, on the host unless out_on_device. */
typedef struct {
  double kernel_ms;        /* device time of the culled sum (CUDA events) */
  double pairs;            /* reference-query pairs evaluated (tile granularity) */
  double full_pairs;       /* pairs of the full sum */
  double max_bound_ratio;  /* max over blocks of skipped bound / smallest block sum */
} bbkde_cull_stats;

BBKDE_API int bbkde_eval_culled(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel, int normalized,
                                double rel_tol, double *out, int out_on_device,
                                bbkde_cull_stats *stats);

/* KernelDensity::eval(queries, rel_err, abs_err[, leaf_nmax, block_size])
 * (KernelDensityImpl.h:624-737, pruning rule :1071-1095): the QUERY set against
 * the REFERENCE set with the reference's combined tolerance. The reference's tree
 * stops refining once a query's bounds are within rel_err relative or abs_err
 * absolute; here the culled sum skips reference tiles whose total bound stays
 * below max(rel_err S, abs_err) / 2, S the smallest near-field density of the
 * query block, so every value f satisfies |out - f| <= max(rel_err f, abs_err) / 2
 * plus the FP32-compensated arithmetic error. abs_err is in normalised density
 * units (the reference divides it by C(h) for its unnormalised sums) and applies
 * as given when normalized = 0 too. 0 <= rel_err < 1, abs_err >= 0 (both 0: every
 * tile that does not flush to zero is summed). Query order is preserved (the
 * reference returns its queries in Kd-tree order). stats->max_bound_ratio is the
 * worst skipped bound over the allowance max(rel_err S, abs_err) (at most 1/2).
 * Kernels as bbkde_eval_culled. */
BBKDE_API int bbkde_eval_tol(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel, int normalized,
                             double rel_err, double abs_err, double *out, int out_on_device,
                             bbkde_cull_stats *stats);

/* A regular 2-D grid: point (i, j), 0 <= i < nx, 0 <= j < ny, at
 * (x0 + i (x1 - x0) / nx, y0 + j (y1 - y0) / ny) (end points excluded, the
 * reference's test grid, test/kde_test_utils.h:97-123); results row-major,
 * index j * nx + i. */
typedef struct {
  int64_t nx, ny;
  double x0, x1, y0, y1;
} bbkde_grid;

enum {
  BBKDE_GRID_EXACT = 0,      /* the exact sum at every point */
  BBKDE_GRID_SURROGATE = 1,  /* network value, held-out probes, exact fallback */
  BBKDE_GRID_ANCHORED = 2    /* network + residual measured exactly at the tiles' first
                                points (anchors), interpolated between them */
};

typedef struct {
  int mode;          /* BBKDE_GRID_* */
  int tile;          /* decision tile edge in grid points: 16 or 32 */
  int probes;        /* held-out probes per tile, judged with the tile's interpolant:
                        1 (centre), 5 (+ edge midpoints, shared with the neighbours)
                        or 9 (+ quarter points); 0 = automatic: 5 while a tile spans
                        at most 0.75 narrowest kernel widths (h times the smallest
                        abw of the reference set), else 9 -- the setting that holds
                        the 1e-3 error bar at every point in the tests. Anchors and
                        the first 5 probes are the points of one lattice of pitch
                        tile/2 (grid index units) from the grid's origin, one pitch
                        past its end; the quarter points a second one: each is one
                        exact grid sum. */
  int exact_culled;  /* 1: exact parts use the culled sum; 0: the full direct sum */
  double rel_tol;    /* a tile keeps the prediction only if every probe is within */
  double low_frac;   /* tiles whose smallest predicted density is below low_frac
                        times the grid's largest go exact */
  double cull_rel;   /* bound of the culled sum (e.g. 1e-7) */
  int interp;        /* anchored mode: residual between the anchors, 1 = bilinear over
                        the tile's corners, 3 = bicubic (Catmull-Rom) over the 4 x 4
                        anchors around the tile; 0 = 1 */
  int pair_form;     /* exact sums on grid tiles: 0 = factored over the axes where the
                        kernel allows it (Gaussians, Epanechnikov product: 2T kernel
                        factors per reference on a T x T tile instead of T^2 kernel
                        values); 1 = the pair form everywhere (for comparison) */
  int net_scope;     /* anchored mode with a network: BBKDE_NET_RESCUE (0) = predict
                        first without it (interpolated exact log-density) and run the
                        network only on the tiles whose probes miss, keeping it where
                        its probes pass; BBKDE_NET_EVERYWHERE (1) = network + residual
                        on every point */
  int lattice_tile;  /* tile edge (in lattice points) of the factored exact sums on the
                        anchor/probe lattices: 16 or 32; 0 = automatic: 32 while a
                        32-point lattice tile spans at most 16 narrowest kernel widths,
                        else 16. A larger tile shares each kernel factor among more
                        points but culls over a larger box */
  int tensor_cores;  /* factored sums on 32 x 32 tiles (lattices, exact tiles): 0 =
                        automatic: on the tcgen05 tensor cores (each factor split into
                        two TF32 terms, up to ~1e-6 relative error against FP64) when
                        the sums are culled with cull_rel >= 1e-5, else on the FP32
                        pipe (FP32-compensated); 1 = always the FP32 pipe; 2 = always
                        the tensor cores */
} bbkde_grid_config;

enum { BBKDE_NET_RESCUE = 0, BBKDE_NET_EVERYWHERE = 1 };

typedef struct {
  int64_t tiles, tiles_low, tiles_flagged, tiles_surrogate;
  int64_t exact_points;       /* points evaluated by an exact sum (lattices, fallback) */
  double pairs;               /* reference-query pairs of those sums (tile granularity) */
  double max_probe_err;       /* largest held-out error among tiles that are not low */
  double max_bound_ratio;     /* largest culled-sum bound ratio */
  double ms_total, ms_predict, ms_probe, ms_fallback;   /* device time (CUDA events):
                        predict = the network (every grid point, or in rescue mode
                        the lattice and the missed tiles, with their re-check);
                        probe = exact lattices, residual interpolation and probe
                        check; fallback = exact tiles */
  int64_t probes_used;        /* the probe set the call ran (resolves probes = 0) */
  int64_t lattice_tile_used;  /* the lattice tile the call ran (resolves lattice_tile = 0) */
} bbkde_grid_stats;

/* Normalised density of the REFERENCE set (with its current attributes, e.g.
 * after bbkde_adapt_density) on a dense 2-D grid. In the surrogate modes the
 * network `sur` predicts log-density (natural log of the normalised density,
 * the quantity it was trained on); sur may be NULL in BBKDE_GRID_ANCHORED mode
 * (a zero network: interpolation of the exact log-density between the anchors)
 * and is ignored in BBKDE_GRID_EXACT mode. out_device holds nx * ny doubles in
 * device memory. No reference counterpart. */
BBKDE_API int bbkde_eval_grid(bbkde_ctx *ctx, bbkde_surrogate *sur,
                              const bbkde_kernel_desc *kernel, const bbkde_grid *grid,
                              const bbkde_grid_config *cfg, double *out_device,
                              bbkde_grid_stats *stats);

/* Least-squares cross-validation with numerical integration of f^2
 * (lsq_numint_cross_validate, KernelDensity.h:24-39, KernelDensityImpl.h:14-97):
 * sum over the grid of f(p)^2 dx dy minus twice the weighted leave-one-out density
 * sum of the REFERENCE set. 2-D kernels (Gaussian, Epanechnikov and their
 * products), BBKDE_FP32C only: the grid term is the culled FP32-compensated sum
 * (bound 1e-7 of each value). The reference's tree tolerances and leaf size have
 * no counterpart (the sums are exact). */
BBKDE_API int bbkde_lsq_numint_cv(bbkde_ctx *ctx, const bbkde_kernel_desc *kernel,
                                  const bbkde_grid *grid, int precision, double *cv_out);

/* ---- introspection ------------------------------------------------------- */

/* Device time (ms, CUDA events on the launching stream) and pair count of the
 * most recent pair-sum kernel launch sequence made by this context. */
BBKDE_API int bbkde_last_launch_stats(const bbkde_ctx *ctx, double *kernel_ms, double *pairs,
                            int64_t *launches);

/* Total number of kernels this context has launched since it was created
 * (-1 for a NULL context). */
BBKDE_API int64_t bbkde_launch_count(const bbkde_ctx *ctx);

/* Launch shapes of the FP32 pair-sum kernels (queries per thread x threads per
 * block, and for the Gaussians whether every 4th, 8th, 16th or 32nd reference's exponentials
 * run on the FP32 pipe instead of MUFU.EX2). By default (variant -1) the context
 * autotunes: for problems of at least
 * 2e10 pairs it times every shape on a slice of the problem once per problem
 * class (kernel, dimension, self-evaluation, log2 sizes) and keeps the fastest.
 * A variant in [0, n_variants) forces that shape. No reference counterpart: the
 * reference takes a block_size hint per call (CudaDirectKde.h:83-88). */
BBKDE_API int bbkde_ctx_set_launch_variant(bbkde_ctx *ctx, int variant);
BBKDE_API int bbkde_launch_variants(const bbkde_ctx *ctx, int *n_variants, int *last_variant);

/* ---- allocation-free evaluation ----------------------------------------- */

/* Direct evaluation that allocates no device memory. It has no counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc -- code
 * running inside a host framework that owns every device allocation through its
 * own pool, work issued where new allocations are forbidden or device memory is
 * already exhausted. The caller passes device pointers for all inputs (FP64
 * columns ref_x / ref_y / ref_mass / ref_abw, query_x / query_y; ref_abw may be
 * NULL, the y columns are ignored for dim 1) and for the output out[n_query]
 * (normalized = 1 multiplies by C(h)). The result matches bbkde_eval_range with
 * BBKDE_FP32C over all references and queries to the FP32C tolerance (the
 * reference range may be cut into fewer segments here, so the last FP32 bits of
 * the summation order can differ).
 *
 * Scratch is one fixed 64 MiB array in the library's device image (held by every
 * device that loads the library until the process exits). Problems that do not
 * fit -- 16 B per reference (20 B for product and convolution kernels), 4 B per
 * query coordinate and at least 8 B per query -- are rejected with
 * BBKDE_OUT_OF_RANGE and a message in errbuf (may be NULL), before any work is
 * enqueued. Up to 1,000,000 references with 1,000,000 2-D queries fit.
 *
 * The work is enqueued on `stream` (a cudaStream_t, NULL = legacy default
 * stream) and the call returns without waiting for it. All calls share the one
 * scratch array, so calls whose GPU work can overlap (different streams, or
 * different host threads without ordering) race and corrupt each other's
 * results; order them on one stream. Every call resolves the array's device
 * address in the current context (cudaGetSymbolAddress). CUDA loads a library's
 * device code lazily, so the first call on a device is the one that places the
 * 64 MiB array in that device's memory; that first call must come before any
 * stream capture and before device memory runs out. A call with n_query = 0 does
 * only this (no work is enqueued), so make one such call per device at set-up,
 * with that device current. Every scratch entry a call reads is written earlier
 * in the same call, so nothing is cleared. */
BBKDE_API int bbkde_eval_noalloc(const bbkde_kernel_desc *kernel, int64_t n_ref,
                                 const double *ref_x, const double *ref_y,
                                 const double *ref_mass, const double *ref_abw,
                                 int64_t n_query, const double *query_x,
                                 const double *query_y, int normalized, double *out,
                                 void *stream, char *errbuf, int64_t errbuf_len);

/* Number of SMs and the device's ordinal (for callers that size their work). */
BBKDE_API int bbkde_device_info(const bbkde_ctx *ctx, int *sm_count, int *device);

#ifdef __cplusplus
}
#endif

#endif /* BBKDE_H_ */
