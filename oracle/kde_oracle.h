/* Test infrastructure, not product code.
 *
 * FP64 CPU restatement of bbrcit_kde's direct kernel-density path, used as the
 * checker for the CUDA library: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it. It is pinned against the reference's
 * own code (oracle/_ref, built from the reference headers) and against the
 * committed golden vectors under tests/golden/.
 *
 * Kernel kinds and their numbering match include/bbkde.h.
 */
#ifndef KDE_ORACLE_H_
#define KDE_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C(h) of the kernel, as the reference computes it (include/Kernels/KernelTraits.h). */
double kde_oracle_normalization(int kind, int dim, const double *h);

/* U(q, r; h*a) for one pair (coords of length dim). */
double kde_oracle_unnormalized(int kind, int dim, const double *h, const double *q,
                               const double *r, double a, int gauss_conv_quirk);

/* out[i] = [C(h) *] sum_j mass[j] * U(q_i, r_j; h*abw[j]) over all n references.
 * abw may be NULL (all ones). Multi-threaded over queries when nthreads > 1. */
int kde_oracle_direct(int kind, int dim, const double *h, int64_t n, const double *r,
                      const double *mass, const double *abw, int64_t m, const double *q,
                      int normalized, int gauss_conv_quirk, double *out, int nthreads);

/* Self-evaluation: out[i] = C * sum_{j != i} mass[j] U(r_i, r_j) when exclude_self,
 * or the full all-pairs sum (self term included) otherwise. */
int kde_oracle_self(int kind, int dim, const double *h, int64_t n, const double *r,
                    const double *mass, const double *abw, int exclude_self,
                    int gauss_conv_quirk, double *out, int nthreads);

/* Weight normalisation and masses (KernelDensityImpl.h:430-455):
 * w_out = w / sum(w); mass_out = w_out * abw^-dim (abw NULL -> 1). */
int kde_oracle_init_attributes(int dim, int64_t n, const double *w, const double *abw,
                               double *w_out, double *mass_out);

/* Adaptive pilot (KernelDensityImpl.h:291-359) over exact direct sums:
 * pilot_i = C * sum_j w_j U(r_i, r_j; h)  (self term included),
 * g = exp(sum_i w_i log pilot_i), abw_i = (pilot_i / g)^-alpha,
 * mass_i = w_i * abw_i^-dim. w must already be normalised. */
int kde_oracle_adapt(int kind, int dim, const double *h, int64_t n, const double *r,
                     const double *w, double alpha, double *pilot_out, double *abw_out,
                     double *mass_out, double *g_out, int nthreads);

/* Leave-one-out likelihood CV (KernelDensityImpl.h:215-252):
 * sum_i w_i log(f_i - mass_i C), where f_i is the all-pairs self sum.
 * loo_mode 0: subtract the self term as the reference does; 1: exclude j == i. */
int kde_oracle_likelihood_cv(int kind, int dim, const double *h, int64_t n,
                             const double *r, const double *w, const double *mass,
                             const double *abw, int loo_mode, double *cv_out, int nthreads);

/* Least-squares CV, convolution form (KernelDensityImpl.h:142-209):
 * sum_i w_i fconv_i - 2 sum_i w_i (f_i - mass_i C). conv_kind is the kernel's
 * convolution kernel (ConvKernelAssociator.h). */
int kde_oracle_lsq_conv_cv(int kind, int conv_kind, int dim, const double *h, int64_t n,
                           const double *r, const double *w, const double *mass,
                           const double *abw, int loo_mode, int gauss_conv_quirk,
                           double *cv_out, int nthreads);

/* Least-squares CV with numerical integration (KernelDensityImpl.h:14-97), 2-D:
 * sum over the steps_x x steps_y grid (x0 + i (x1 - x0) / steps_x, ...; end points
 * excluded) of f^2 dx dy, minus 2 sum_i w_i (f_i - mass_i C). */
int kde_oracle_lsq_numint_cv(int kind, const double *h, int64_t n, const double *r,
                             const double *w, const double *mass, const double *abw,
                             double x0, double x1, int steps_x, double y0, double y1,
                             int steps_y, int loo_mode, double *cv_out, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
