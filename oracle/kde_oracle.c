/* Test infrastructure, not product code: the FP64 CPU oracle.
 *
 * A plain-C restatement of bbrcit_kde's direct kernel-density path. Each function
 * cites the reference file:line it follows (paths relative to the reference
 * project root). Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load this library; the CUDA library never calls it.
 *
 * Parity pin: tests/test_oracle_cpu.py checks every function here against the
 * reference's own code (oracle/_ref/libkde_ref.so, built from the reference
 * headers) and against the committed golden vectors in tests/golden/.
 */
#define _GNU_SOURCE
#include "kde_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

enum {
  K_GAUSS = 0, K_EPAN = 1, K_GAUSS_PROD2D = 2, K_EPAN_PROD2D = 3,
  K_GAUSS_PROD_CONV2D = 4, K_EPAN_PROD_CONV2D = 5, K_GAUSS_CONV1D = 6, K_EPAN_CONV1D = 7
};

/* Normalisation constants: include/Kernels/KernelTraits.h
 *   Gaussian 1-D  :143-145  0.3989422804014326779 / h, with h passed as float
 *   Gaussian 2-D  :157-159  0.1591549430918953357 / (h*h)
 *   Epan 1-D      :53-55    0.75 / h
 *   Epan 2-D      :81-83    0.6366197723675813431 / (h*h)
 *   GaussProd2d   :205-207  0.1591549430918953357 / (hx*hy)
 *   EpanProd2d    :250-252  0.5625 / (hx*hy)
 *   EpanConv1d    :299-301  0.6 / h
 *   EpanProdConv2d:349-351  0.36 / (hx*hy)
 *   GaussConv1d   :396-398  0.2820947917738781434 / h
 *   GaussProdConv2d:440-442 0.0795774715459476678 / (hx*hy) */
double kde_oracle_normalization(int kind, int dim, const double *h) {
  switch (kind) {
    case K_GAUSS:
      if (dim == 1) return 0.3989422804014326779 / (double)(float)h[0];
      return 0.1591549430918953357 / (h[0] * h[0]);
    case K_EPAN:
      if (dim == 1) return 0.75 / h[0];
      return 0.6366197723675813431 / (h[0] * h[0]);
    case K_GAUSS_PROD2D: return 0.1591549430918953357 / (h[0] * h[1]);
    case K_EPAN_PROD2D: return 0.5625 / (h[0] * h[1]);
    case K_GAUSS_PROD_CONV2D: return 0.0795774715459476678 / (h[0] * h[1]);
    case K_EPAN_PROD_CONV2D: return 0.36 / (h[0] * h[1]);
    case K_GAUSS_CONV1D: return 0.2820947917738781434 / h[0];
    case K_EPAN_CONV1D: return 0.6 / h[0];
  }
  return 0.0;
}

/* (2-|u|)^3 (u^2 + 6|u| + 4) / 32 on |u| < 2: KernelTraits.h:303-307, :353-357. */
static double epan_conv_poly(double u) {
  u = fabs(u);
  double cubic = fmax(2.0 - u, 0.0);
  return 0.03125 * cubic * cubic * cubic * (u * u + 6.0 * u + 4.0);
}

/* U(q, r; h*a), following the generic point_arg_eval / unnormalized_eval of each
 * kernel (the path DecoratedPoint<> coordinates take on the CPU):
 *   GaussianKernel.h:129-142 + KernelTraits.h:147-149/161-163 exp(-0.5 arg)
 *   EpanechnikovKernel.h:133-146 + KernelTraits.h:57-59/85-87 max(1-arg,0)
 *   GaussianProductKernel2d.h:144-150 + KernelTraits.h:210-212
 *   EpanechnikovProductKernel2d.h:140-145 + KernelTraits.h:254-256
 *   GaussianProductConvKernel2d.h:139-143 + KernelTraits.h:444-446. The reference's
 *     double specialisation evaluates exp(-0.5 arg), while the generic template and
 *     the kernel's own documentation give exp(-0.25 arg) (KernelTraits.h:418-420).
 *     gauss_conv_quirk != 0 reproduces the reference; 0 uses -0.25.
 *   EpanechnikovProductConvKernel2d.h:131-136 + KernelTraits.h:353-357
 *   GaussianConvKernel1d.h:112-121 + KernelTraits.h:400-402 exp(-0.25 arg)
 *   EpanechnikovConvKernel1d.h:111-113 + KernelTraits.h:303-307 */
double kde_oracle_unnormalized(int kind, int dim, const double *h, const double *q,
                               const double *r, double a, int gauss_conv_quirk) {
  switch (kind) {
    case K_GAUSS: {
      double s = 0.0;
      for (int d = 0; d < dim; ++d) { double df = q[d] - r[d]; s += df * df; }
      return exp(-0.5 * (s / (h[0] * h[0] * a * a)));
    }
    case K_EPAN: {
      double s = 0.0;
      for (int d = 0; d < dim; ++d) { double df = q[d] - r[d]; s += df * df; }
      return fmax(1.0 - s / (h[0] * h[0] * a * a), 0.0);
    }
    case K_GAUSS_PROD2D: {
      double arg = (q[0] - r[0]) * (q[0] - r[0]) / (h[0] * h[0] * a * a) +
                   (q[1] - r[1]) * (q[1] - r[1]) / (h[1] * h[1] * a * a);
      return exp(-0.5 * arg);
    }
    case K_EPAN_PROD2D: {
      double ax = (q[0] - r[0]) * (q[0] - r[0]) / (h[0] * h[0] * a * a);
      double ay = (q[1] - r[1]) * (q[1] - r[1]) / (h[1] * h[1] * a * a);
      return fmax(1.0 - ax, 0.0) * fmax(1.0 - ay, 0.0);
    }
    case K_GAUSS_PROD_CONV2D: {
      double arg = (q[0] - r[0]) * (q[0] - r[0]) / (h[0] * h[0] * a * a) +
                   (q[1] - r[1]) * (q[1] - r[1]) / (h[1] * h[1] * a * a);
      return exp((gauss_conv_quirk ? -0.5 : -0.25) * arg);
    }
    case K_EPAN_PROD_CONV2D:
      return epan_conv_poly((q[0] - r[0]) / (h[0] * a)) *
             epan_conv_poly((q[1] - r[1]) / (h[1] * a));
    case K_GAUSS_CONV1D: {
      double arg = (q[0] - r[0]) * (q[0] - r[0]) / (h[0] * h[0] * a * a);
      return exp(-0.25 * arg);
    }
    case K_EPAN_CONV1D:
      return epan_conv_poly((q[0] - r[0]) / (h[0] * a));
  }
  return 0.0;
}

/* ---- threaded direct sums ------------------------------------------------ */

typedef struct {
  int kind, dim; const double *h;
  int64_t n; const double *r; const double *mass; const double *abw;
  const double *q; double *out; double c;
  int self_mode;   /* 0: plain queries, 1: self-eval incl. self, 2: self-eval excl. self */
  int quirk;
  int64_t lo, hi;
} job_t;

/* Serial double loop of KernelDensity::direct_eval (KernelDensityImpl.h:1157-1173). */
static void *direct_worker(void *arg) {
  job_t *j = (job_t *)arg;
  for (int64_t i = j->lo; i < j->hi; ++i) {
    const double *qi = j->q + i * j->dim;
    double total = 0.0;
    for (int64_t k = 0; k < j->n; ++k) {
      if (j->self_mode == 2 && k == i) continue;
      double a = j->abw ? j->abw[k] : 1.0;
      total += j->mass[k] * kde_oracle_unnormalized(j->kind, j->dim, j->h, qi,
                                                    j->r + k * j->dim, a, j->quirk);
    }
    j->out[i] = total * j->c;
  }
  return NULL;
}

static int run_threads(job_t proto, int64_t m, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if (m < 64 || nthreads == 1) {
    proto.lo = 0; proto.hi = m; direct_worker(&proto); return 0;
  }
  pthread_t th[256]; job_t jobs[256]; int live[256];
  int64_t chunk = (m + nthreads - 1) / nthreads;
  int njobs = 0;
  for (int t = 0; t < nthreads; ++t) {
    jobs[t] = proto;
    jobs[t].lo = t * chunk;
    jobs[t].hi = jobs[t].lo + chunk < m ? jobs[t].lo + chunk : m;
    if (jobs[t].lo >= jobs[t].hi) break;
    live[t] = pthread_create(&th[t], NULL, direct_worker, &jobs[t]) == 0;
    if (!live[t]) direct_worker(&jobs[t]);   /* no thread available: run inline */
    ++njobs;
  }
  for (int t = 0; t < njobs; ++t) if (live[t]) pthread_join(th[t], NULL);
  return 0;
}

int kde_oracle_direct(int kind, int dim, const double *h, int64_t n, const double *r,
                      const double *mass, const double *abw, int64_t m, const double *q,
                      int normalized, int gauss_conv_quirk, double *out, int nthreads) {
  if (dim < 1 || dim > 2 || n < 0 || m < 0) return 2;
  job_t j = {kind, dim, h, n, r, mass, abw, q, out,
             normalized ? kde_oracle_normalization(kind, dim, h) : 1.0,
             0, gauss_conv_quirk, 0, 0};
  return run_threads(j, m, nthreads);
}

int kde_oracle_self(int kind, int dim, const double *h, int64_t n, const double *r,
                    const double *mass, const double *abw, int exclude_self,
                    int gauss_conv_quirk, double *out, int nthreads) {
  if (dim < 1 || dim > 2 || n < 0) return 2;
  job_t j = {kind, dim, h, n, r, mass, abw, r, out,
             kde_oracle_normalization(kind, dim, h),
             exclude_self ? 2 : 1, gauss_conv_quirk, 0, 0};
  return run_threads(j, n, nthreads);
}

/* KernelDensityImpl.h:430-455: normalize_weights then mass = w * pow(abw, -D). */
int kde_oracle_init_attributes(int dim, int64_t n, const double *w, const double *abw,
                               double *w_out, double *mass_out) {
  double total = 0.0;
  for (int64_t i = 0; i < n; ++i) total += w ? w[i] : 1.0;
  for (int64_t i = 0; i < n; ++i) {
    double wi = (w ? w[i] : 1.0) / total;
    if (w_out) w_out[i] = wi;
    if (mass_out) mass_out[i] = wi * pow(abw ? abw[i] : 1.0, -dim);
  }
  return 0;
}

/* KernelDensityImpl.h:291-359 with the tree self-eval (:319-325) replaced by the
 * exact all-pairs direct sum it approximates (self term included). */
int kde_oracle_adapt(int kind, int dim, const double *h, int64_t n, const double *r,
                     const double *w, double alpha, double *pilot_out, double *abw_out,
                     double *mass_out, double *g_out, int nthreads) {
  if (alpha < 0 || alpha > 1) return 2;                       /* :301-303 */
  double *pilot = pilot_out ? pilot_out : (double *)malloc(sizeof(double) * (size_t)n);
  if (!pilot) return 7;
  /* unadapt_density (:254-273): abw = 1, mass = weight */
  int rc = kde_oracle_self(kind, dim, h, n, r, w, NULL, 0, 1, pilot, nthreads);
  if (rc) { if (!pilot_out) free(pilot); return rc; }
  if (alpha == 0) {                                           /* :311 */
    for (int64_t i = 0; i < n; ++i) { abw_out[i] = 1.0; mass_out[i] = w[i]; }
    if (g_out) *g_out = NAN;
    if (!pilot_out) free(pilot);
    return 0;
  }
  double g = 0.0;                                             /* :330-336 */
  for (int64_t i = 0; i < n; ++i) g += w[i] * log(pilot[i]);
  g = exp(g);
  for (int64_t i = 0; i < n; ++i) {                           /* :338-353 */
    double bw = pow(pilot[i] / g, -alpha);
    abw_out[i] = bw;
    mass_out[i] = w[i] * pow(bw, -dim);
  }
  if (g_out) *g_out = g;
  if (!pilot_out) free(pilot);
  return 0;
}

/* KernelDensityImpl.h:215-252. */
int kde_oracle_likelihood_cv(int kind, int dim, const double *h, int64_t n,
                             const double *r, const double *w, const double *mass,
                             const double *abw, int loo_mode, double *cv_out, int nthreads) {
  double *f = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1));
  if (!f) return 7;
  double c = kde_oracle_normalization(kind, dim, h);
  int rc = kde_oracle_self(kind, dim, h, n, r, mass, abw, loo_mode == 1, 1, f, nthreads);
  if (rc) { free(f); return rc; }
  double cv = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double v = f[i];
    if (loo_mode == 0) v -= mass[i] * c;                      /* :244-245 */
    cv += w[i] * log(v);                                      /* :248 */
  }
  *cv_out = cv;
  free(f);
  return 0;
}

/* KernelDensityImpl.h:142-209. */
int kde_oracle_lsq_conv_cv(int kind, int conv_kind, int dim, const double *h, int64_t n,
                           const double *r, const double *w, const double *mass,
                           const double *abw, int loo_mode, int gauss_conv_quirk,
                           double *cv_out, int nthreads) {
  double *f = (double *)malloc(sizeof(double) * (size_t)(n ? n : 1) * 2);
  if (!f) return 7;
  double *fc = f + n;
  double c = kde_oracle_normalization(kind, dim, h);
  int rc = kde_oracle_self(kind, dim, h, n, r, mass, abw, loo_mode == 1, 1, f, nthreads);
  if (!rc) rc = kde_oracle_self(conv_kind, dim, h, n, r, mass, abw, 0, gauss_conv_quirk,
                                fc, nthreads);
  if (rc) { free(f); return rc; }
  double llo = 0.0, sq = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double v = f[i];
    if (loo_mode == 0) v -= mass[i] * c;                      /* :176-177 */
    llo += w[i] * v;                                          /* :180 */
    sq += w[i] * fc[i];                                       /* :201-204 */
  }
  *cv_out = sq - 2 * llo;                                     /* :207 */
  free(f);
  return 0;
}

/* KernelDensityImpl.h:14-97: LOO term over the self sums (:47-60), square
 * integral over the grid (:66-94; grid built at :69-75 with y outer, x inner). */
int kde_oracle_lsq_numint_cv(int kind, const double *h, int64_t n, const double *r,
                             const double *w, const double *mass, const double *abw,
                             double x0, double x1, int steps_x, double y0, double y1,
                             int steps_y, int loo_mode, double *cv_out, int nthreads) {
  const int64_t m = (int64_t)steps_x * steps_y;
  double *f = (double *)malloc(sizeof(double) * (size_t)((n ? n : 1) + m + 2 * m));
  if (!f) return 7;
  double *fg = f + (n ? n : 1), *q = fg + m;
  const double c = kde_oracle_normalization(kind, 2, h);
  int rc = kde_oracle_self(kind, 2, h, n, r, mass, abw, loo_mode == 1, 1, f, nthreads);
  const double dx = (x1 - x0) / steps_x, dy = (y1 - y0) / steps_y;
  for (int j = 0; j < steps_y; ++j)
    for (int i = 0; i < steps_x; ++i) {
      q[2 * ((int64_t)j * steps_x + i)] = x0 + i * dx;
      q[2 * ((int64_t)j * steps_x + i) + 1] = y0 + j * dy;
    }
  if (!rc) rc = kde_oracle_direct(kind, 2, h, n, r, mass, abw, m, q, 1, 1, fg, nthreads);
  if (rc) { free(f); return rc; }
  double llo = 0.0, sq = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double v = f[i];
    if (loo_mode == 0) v -= mass[i] * c;                      /* :55-56 */
    llo += w[i] * v;                                          /* :59 */
  }
  for (int64_t k = 0; k < m; ++k) sq += fg[k] * fg[k] * dx * dy;   /* :86-92 */
  *cv_out = sq - 2 * llo;                                     /* :95 */
  free(f);
  return 0;
}
