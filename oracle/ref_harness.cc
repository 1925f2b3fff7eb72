// Test infrastructure, not product code: a C-ABI shim around the reference
// implementation (bbrcit_kde's header-only KernelDensity<> templates), compiled
// from the reference's own headers by oracle/Makefile into oracle/_ref/.
//
// It is used for three things only:
//   * pinning the C restatement in oracle/kde_oracle.c (tests/test_oracle_cpu.py),
//   * generating the committed golden vectors (tests/golden/make_golden.py),
//   * timing the reference CPU path (bench.py cpu_baseline / --impl reference).
// Nothing in the product library links or calls this file.
//
// Every entry point builds a KernelDensity<D, Kernel<double>, double> exactly as
// a user of the reference would: points are DecoratedPoint{{coords},{weight}},
// the constructor normalises weights and builds the Kd-tree
// (include/KernelDensityImpl.h:388-398, include/Kdtree.h:340-390), and the
// requested method is called through the public API.
//
// Direct evaluation is spread over host threads with std::thread chunks over
// queries: KernelDensity::direct_eval(DataPointType&) is const and writes only
// to its argument (include/KernelDensityImpl.h:1148-1154), so disjoint query
// chunks are independent. The reference itself demonstrates this pattern in
// test/test_kde_cppthread.cc:91-106.

#include <cmath>
#include <cstdint>
#include <random>  // the reference headers use std:: distributions without including it
#include <cstring>
#include <iostream>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

#include <KernelDensity.h>
#include <MarginalDensityAssociator.h>
#include <Kernels/EpanechnikovKernel.h>
#include <Kernels/EpanechnikovProductKernel2d.h>
#include <Kernels/EpanechnikovProductConvKernel2d.h>
#include <Kernels/EpanechnikovConvKernel1d.h>
#include <Kernels/GaussianKernel.h>
#include <Kernels/GaussianProductKernel2d.h>
#include <Kernels/GaussianProductConvKernel2d.h>
#include <Kernels/GaussianConvKernel1d.h>

namespace {

using namespace bbrcit;

// Kernel kinds, numbered as in include/bbkde.h.
enum Kind {
  GAUSS = 0, EPAN = 1, GAUSS_PROD2D = 2, EPAN_PROD2D = 3,
  GAUSS_PROD_CONV2D = 4, EPAN_PROD_CONV2D = 5, GAUSS_CONV1D = 6, EPAN_CONV1D = 7
};

// The reference reports every bound wider than the requested tolerance on
// std::cerr (KernelDensityImpl.h:1113-1143), at rel = abs = 0 for nearly every
// point; this mutes it for the duration of one call.
struct MuteCerr {
  // Calls may run on several host threads at once (the CPU baselines): the first
  // one in mutes the stream, the last one out restores it.
  static std::mutex &mu() {
    static std::mutex m;
    return m;
  }
  static int &depth() {
    static int d = 0;
    return d;
  }
  static std::streambuf *&saved() {
    static std::streambuf *b = nullptr;
    return b;
  }
  MuteCerr() {
    std::lock_guard<std::mutex> lock(mu());
    if (depth()++ == 0) saved() = std::cerr.rdbuf(nullptr);
  }
  ~MuteCerr() {
    std::lock_guard<std::mutex> lock(mu());
    if (--depth() == 0) {
      std::cerr.rdbuf(saved());
      std::cerr.clear();
    }
  }
};

template <typename K> void set_bw(K &k, const double *h) { k.set_bandwidth(h[0]); }
template <> void set_bw(GaussianProductKernel2d<double> &k, const double *h) { k.set_bandwidths(h[0], h[1]); }
template <> void set_bw(EpanechnikovProductKernel2d<double> &k, const double *h) { k.set_bandwidths(h[0], h[1]); }
template <> void set_bw(GaussianProductConvKernel2d<double> &k, const double *h) { k.set_bandwidths(h[0], h[1]); }
template <> void set_bw(EpanechnikovProductConvKernel2d<double> &k, const double *h) { k.set_bandwidths(h[0], h[1]); }
// The 1-D convolution kernels only expose a constructor bandwidth.
template <> void set_bw(GaussianConvKernel1d<double> &k, const double *h) { k = GaussianConvKernel1d<double>(h[0]); }
template <> void set_bw(EpanechnikovConvKernel1d<double> &k, const double *h) { k = EpanechnikovConvKernel1d<double>(h[0]); }

template <int D, typename K>
using KdeT = KernelDensity<D, K, double>;

template <int D, typename K>
std::vector<typename KdeT<D, K>::DataPointType>
make_points(int64_t n, const double *xy, const double *w) {
  using P = typename KdeT<D, K>::DataPointType;
  std::vector<P> pts;
  pts.reserve(n);
  for (int64_t i = 0; i < n; ++i) {
    P p;
    for (int d = 0; d < D; ++d) p[d] = xy[i * D + d];
    p.attributes() = AdaKdeAttributes<double>(w ? w[i] : 1.0);
    pts.push_back(p);
  }
  return pts;
}

template <int D, typename K>
void threaded_direct_eval(const KdeT<D, K> &kde, int64_t m, const double *q,
                          double *out, int nthreads) {
  using P = typename KdeT<D, K>::DataPointType;
  if (nthreads < 1) nthreads = 1;
  auto work = [&](int64_t lo, int64_t hi) {
    P p;
    for (int64_t i = lo; i < hi; ++i) {
      for (int d = 0; d < D; ++d) p[d] = q[i * D + d];
      out[i] = kde.direct_eval(p);
    }
  };
  if (nthreads == 1 || m < 64) { work(0, m); return; }
  std::vector<std::thread> th;
  int64_t chunk = (m + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    int64_t lo = t * chunk, hi = std::min<int64_t>(m, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back(work, lo, hi);
  }
  for (auto &t : th) t.join();
}

template <int D, typename K>
void export_tree(const KdeT<D, K> &kde, double *xy, double *w, double *mass,
                 double *abw, int64_t *n_out) {
  const auto &pts = kde.points();
  if (n_out) *n_out = (int64_t)pts.size();
  for (size_t i = 0; i < pts.size(); ++i) {
    if (xy) for (int d = 0; d < D; ++d) xy[i * D + d] = pts[i][d];
    if (w) w[i] = pts[i].attributes().weight();
    if (mass) mass[i] = pts[i].attributes().mass();
    if (abw) abw[i] = pts[i].attributes().abw();
  }
}

// One request covering every method the harness exposes.
struct Req {
  int kind, dim;
  const double *h;
  int64_t n; const double *xy; const double *w;
  double alpha; double rel, abs;       // alpha < 0: no adaptation
  int64_t m; const double *q; double *out;
  double *tree_xy, *tree_w, *tree_mass, *tree_abw; int64_t *n_tree;
  double *lik_cv, *lsq_cv;              // CV outputs (may be null)
  int nthreads;
};

template <int D, typename K>
int run(const Req &r) {
  MuteCerr mute;
  KdeT<D, K> kde(make_points<D, K>(r.n, r.xy, r.w), 2);
  set_bw(kde.kernel(), r.h);
  if (r.alpha >= 0) kde.adapt_density(r.alpha, r.rel, r.abs);
  if (r.m > 0 && r.q && r.out) threaded_direct_eval(kde, r.m, r.q, r.out, r.nthreads);
  export_tree(kde, r.tree_xy, r.tree_w, r.tree_mass, r.tree_abw, r.n_tree);
  if (r.lik_cv) *r.lik_cv = kde.likelihood_cross_validate(r.rel, r.abs);
  return 0;
}

// LSQ convolution CV is only defined for kernels with a ConvKernelAssociator
// specialisation (include/Kernels/ConvKernelAssociator.h:22-84).
template <int D, typename K>
int run_lsq(const Req &r) {
  MuteCerr mute;
  KdeT<D, K> kde(make_points<D, K>(r.n, r.xy, r.w), 2);
  set_bw(kde.kernel(), r.h);
  if (r.alpha >= 0) kde.adapt_density(r.alpha, r.rel, r.abs);
  *r.lsq_cv = kde.lsq_convolution_cross_validate(r.rel, r.abs);
  return 0;
}

int dispatch(const Req &r) {
  if (r.dim == 1) {
    switch (r.kind) {
      case GAUSS: return run<1, GaussianKernel<1, double>>(r);
      case EPAN: return run<1, EpanechnikovKernel<1, double>>(r);
      case GAUSS_CONV1D: return run<1, GaussianConvKernel1d<double>>(r);
      case EPAN_CONV1D: return run<1, EpanechnikovConvKernel1d<double>>(r);
    }
  } else if (r.dim == 2) {
    switch (r.kind) {
      case GAUSS: return run<2, GaussianKernel<2, double>>(r);
      case EPAN: return run<2, EpanechnikovKernel<2, double>>(r);
      case GAUSS_PROD2D: return run<2, GaussianProductKernel2d<double>>(r);
      case EPAN_PROD2D: return run<2, EpanechnikovProductKernel2d<double>>(r);
      case GAUSS_PROD_CONV2D: return run<2, GaussianProductConvKernel2d<double>>(r);
      case EPAN_PROD_CONV2D: return run<2, EpanechnikovProductConvKernel2d<double>>(r);
    }
  }
  return 5;  // unsupported
}

// Free function lsq_numint_cross_validate (KernelDensity.h:24-39,
// KernelDensityImpl.h:14-97) on 2-D kernels.
struct NumintReq {
  double x0, x1, y0, y1;
  int sx, sy;
};

template <typename K>
int run_numint(const Req &r, const NumintReq &g) {
  MuteCerr mute;
  KdeT<2, K> kde(make_points<2, K>(r.n, r.xy, r.w), 2);
  set_bw(kde.kernel(), r.h);
  if (r.alpha >= 0) kde.adapt_density(r.alpha, r.rel, r.abs);
  *r.lsq_cv = lsq_numint_cross_validate(kde, g.x0, g.x1, g.sx, g.y0, g.y1, g.sy, r.rel, r.abs,
                                        2);
  return 0;
}

int dispatch_numint(const Req &r, const NumintReq &g) {
  switch (r.kind) {
    case GAUSS: return run_numint<GaussianKernel<2, double>>(r, g);
    case EPAN: return run_numint<EpanechnikovKernel<2, double>>(r, g);
    case GAUSS_PROD2D: return run_numint<GaussianProductKernel2d<double>>(r, g);
    case EPAN_PROD2D: return run_numint<EpanechnikovProductKernel2d<double>>(r, g);
  }
  return 5;
}

int dispatch_lsq(const Req &r) {
  if (r.dim == 1) {
    switch (r.kind) {
      case GAUSS: return run_lsq<1, GaussianKernel<1, double>>(r);
      case EPAN: return run_lsq<1, EpanechnikovKernel<1, double>>(r);
    }
  } else if (r.dim == 2) {
    switch (r.kind) {
      case GAUSS_PROD2D: return run_lsq<2, GaussianProductKernel2d<double>>(r);
      case EPAN_PROD2D: return run_lsq<2, EpanechnikovProductKernel2d<double>>(r);
    }
  }
  return 5;
}

// KernelDensity::eval(std::vector<DataPointType>&, rel_err, abs_err, leaf_nmax)
// (KernelDensityImpl.h:624-651): the reference's dual-tree evaluation. The query
// tree reorders the queries and merges exact duplicates, so the returned
// coordinates go to out_q (m_out rows of D) beside their values in out. The
// data points (after an exact adapt_density when alpha >= 0) are exported
// through the tree_* outputs, so that a comparison can evaluate with identical
// attributes.

template <int D, typename K>
int run_tree_eval(const Req &r, double *out_q, int64_t *m_out) {
  using P = typename KdeT<D, K>::DataPointType;
  MuteCerr mute;
  KdeT<D, K> kde(make_points<D, K>(r.n, r.xy, r.w), 2);
  set_bw(kde.kernel(), r.h);
  if (r.alpha >= 0) kde.adapt_density(r.alpha, 0.0, 0.0);
  std::vector<P> q;
  q.reserve(r.m);
  for (int64_t i = 0; i < r.m; ++i) {
    P p;
    for (int d = 0; d < D; ++d) p[d] = r.q[i * D + d];
    q.push_back(p);
  }
  kde.eval(q, r.rel, r.abs, 32);
  for (size_t i = 0; i < q.size(); ++i) {
    for (int d = 0; d < D; ++d) out_q[i * D + d] = q[i][d];
    r.out[i] = q[i].attributes().value();
  }
  *m_out = (int64_t)q.size();
  export_tree(kde, r.tree_xy, r.tree_w, r.tree_mass, r.tree_abw, r.n_tree);
  return 0;
}

int dispatch_tree_eval(const Req &r, double *out_q, int64_t *m_out) {
  if (r.dim == 1) {
    switch (r.kind) {
      case GAUSS: return run_tree_eval<1, GaussianKernel<1, double>>(r, out_q, m_out);
      case EPAN: return run_tree_eval<1, EpanechnikovKernel<1, double>>(r, out_q, m_out);
    }
  } else if (r.dim == 2) {
    switch (r.kind) {
      case GAUSS: return run_tree_eval<2, GaussianKernel<2, double>>(r, out_q, m_out);
      case EPAN: return run_tree_eval<2, EpanechnikovKernel<2, double>>(r, out_q, m_out);
      case GAUSS_PROD2D:
        return run_tree_eval<2, GaussianProductKernel2d<double>>(r, out_q, m_out);
      case EPAN_PROD2D:
        return run_tree_eval<2, EpanechnikovProductKernel2d<double>>(r, out_q, m_out);
    }
  }
  return 5;
}

// MarginalDensityAssociator<KernelDensity<2, K, double>>::marginal_density(kde,
// dim_idx) (MarginalDensityAssociator.h:95-118) of the (optionally adapted)
// 2-D density, then direct_eval of the 1-D marginal at m queries. The marginal's
// own points (its Kd-tree order, duplicates merged) are exported through the
// tree_* outputs (coordinate, weight, mass, abw).
template <typename K>
int run_marginal(const Req &r, int dim_idx) {
  using Assoc = MarginalDensityAssociator<KdeT<2, K>>;
  MuteCerr mute;
  KdeT<2, K> kde(make_points<2, K>(r.n, r.xy, r.w), 2);
  set_bw(kde.kernel(), r.h);
  if (r.alpha >= 0) kde.adapt_density(r.alpha, r.rel, r.abs);
  typename Assoc::MarginalDensityType m = Assoc::marginal_density(kde, (size_t)dim_idx);
  if (r.m > 0 && r.q && r.out) threaded_direct_eval(m, r.m, r.q, r.out, r.nthreads);
  export_tree(m, r.tree_xy, r.tree_w, r.tree_mass, r.tree_abw, r.n_tree);
  return 0;
}

// A KernelDensity kept alive across calls, for timing repeated direct_eval
// batches without rebuilding the Kd-tree (bench.py's CPU baseline).
struct Handle {
  virtual ~Handle() {}
  virtual void direct(int64_t m, const double *q, double *out, int nthreads) const = 0;
};

template <int D, typename K>
struct HandleT : Handle {
  KdeT<D, K> kde;
  HandleT(int64_t n, const double *xy, const double *w, const double *h)
      : kde(make_points<D, K>(n, xy, w), 2) { set_bw(kde.kernel(), h); }
  void direct(int64_t m, const double *q, double *out, int nthreads) const override {
    threaded_direct_eval(kde, m, q, out, nthreads);
  }
};

Handle *make_handle(int kind, int dim, const double *h, int64_t n, const double *xy,
                    const double *w) {
  if (dim == 1) {
    switch (kind) {
      case GAUSS: return new HandleT<1, GaussianKernel<1, double>>(n, xy, w, h);
      case EPAN: return new HandleT<1, EpanechnikovKernel<1, double>>(n, xy, w, h);
    }
  } else if (dim == 2) {
    switch (kind) {
      case GAUSS: return new HandleT<2, GaussianKernel<2, double>>(n, xy, w, h);
      case EPAN: return new HandleT<2, EpanechnikovKernel<2, double>>(n, xy, w, h);
      case GAUSS_PROD2D: return new HandleT<2, GaussianProductKernel2d<double>>(n, xy, w, h);
      case EPAN_PROD2D: return new HandleT<2, EpanechnikovProductKernel2d<double>>(n, xy, w, h);
    }
  }
  return nullptr;
}

}  // namespace

extern "C" {

void *ref_kde_create(int kind, int dim, const double *h, int64_t n, const double *xy,
                     const double *w) {
  try { return make_handle(kind, dim, h, n, xy, w); } catch (...) { return nullptr; }
}

int ref_kde_direct(void *handle, int64_t m, const double *q, double *out, int nthreads) {
  if (!handle) return 2;
  static_cast<Handle *>(handle)->direct(m, q, out, nthreads);
  return 0;
}

void ref_kde_destroy(void *handle) { delete static_cast<Handle *>(handle); }

// Direct evaluation at `m` queries, optionally after adapt_density(alpha, rel, abs)
// (alpha < 0 skips adaptation). Also exports the Kd-tree ordered data points
// (coords, normalised weight, mass, abw) when the tree_* pointers are non-null.
int ref_kde_eval(int kind, int dim, const double *h, int64_t n, const double *xy,
                 const double *w, double alpha, double rel, double abs, int64_t m,
                 const double *q, double *out, double *tree_xy, double *tree_w,
                 double *tree_mass, double *tree_abw, int64_t *n_tree, int nthreads) {
  try {
    Req r{kind, dim, h, n, xy, w, alpha, rel, abs, m, q, out,
          tree_xy, tree_w, tree_mass, tree_abw, n_tree, nullptr, nullptr, nthreads};
    return dispatch(r);
  } catch (const std::invalid_argument &) { return 2; }
  catch (...) { return 9; }
}

// KernelDensity::likelihood_cross_validate(rel, abs) after optional adaptation.
int ref_kde_likelihood_cv(int kind, int dim, const double *h, int64_t n,
                          const double *xy, const double *w, double alpha,
                          double rel, double abs, double *cv) {
  try {
    Req r{kind, dim, h, n, xy, w, alpha, rel, abs, 0, nullptr, nullptr,
          nullptr, nullptr, nullptr, nullptr, nullptr, cv, nullptr, 1};
    return dispatch(r);
  } catch (const std::invalid_argument &) { return 2; }
  catch (...) { return 9; }
}

// KernelDensity::lsq_convolution_cross_validate(rel, abs).
int ref_kde_lsq_conv_cv(int kind, int dim, const double *h, int64_t n,
                        const double *xy, const double *w, double alpha,
                        double rel, double abs, double *cv) {
  try {
    Req r{kind, dim, h, n, xy, w, alpha, rel, abs, 0, nullptr, nullptr,
          nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, cv, 1};
    return dispatch_lsq(r);
  } catch (const std::invalid_argument &) { return 2; }
  catch (...) { return 9; }
}

// lsq_numint_cross_validate(kde, x0, x1, sx, y0, y1, sy, rel, abs, leaf_nmax).
int ref_kde_lsq_numint_cv(int kind, const double *h, int64_t n, const double *xy,
                          const double *w, double alpha, double x0, double x1, int sx,
                          double y0, double y1, int sy, double rel, double abs, double *cv) {
  try {
    Req r{kind, 2, h, n, xy, w, alpha, rel, abs, 0, nullptr, nullptr,
          nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, cv, 1};
    NumintReq g{x0, x1, y0, y1, sx, sy};
    return dispatch_numint(r, g);
  } catch (const std::invalid_argument &) { return 2; }
  catch (...) { return 9; }
}

// KernelDensity::eval(queries, rel_err, abs_err) (see run_tree_eval), after an
// exact adapt_density(alpha, 0, 0) when alpha >= 0. Exports the data points in
// tree order like ref_kde_eval. Returns 2 on invalid arguments, 5 unsupported.
int ref_kde_tree_eval(int kind, int dim, const double *h, int64_t n, const double *xy,
                      const double *w, double alpha, double rel, double abs, int64_t m,
                      const double *q, double *out_q, double *out, int64_t *m_out,
                      double *tree_xy, double *tree_w, double *tree_mass, double *tree_abw,
                      int64_t *n_tree) {
  try {
    Req r{kind, dim, h, n, xy, w, alpha, rel, abs, m, q, out,
          tree_xy, tree_w, tree_mass, tree_abw, n_tree, nullptr, nullptr, 1};
    return dispatch_tree_eval(r, out_q, m_out);
  } catch (const std::invalid_argument &) { return 2; }
  catch (...) { return 9; }
}

// The 1-D marginal density of a 2-D product-kernel density (see run_marginal):
// kind GAUSS_PROD2D or EPAN_PROD2D; adapt_density(alpha, rel, abs) first when
// alpha >= 0; direct_eval at m 1-D queries.
int ref_kde_marginal_direct(int kind, const double *h, int64_t n, const double *xy,
                            const double *w, double alpha, double rel, double abs, int dim_idx,
                            int64_t m, const double *q, double *out, double *tree_x,
                            double *tree_w, double *tree_mass, double *tree_abw,
                            int64_t *n_tree, int nthreads) {
  try {
    Req r{kind, 2, h, n, xy, w, alpha, rel, abs, m, q, out,
          tree_x, tree_w, tree_mass, tree_abw, n_tree, nullptr, nullptr, nthreads};
    if (dim_idx != 0 && dim_idx != 1) return 2;
    if (kind == GAUSS_PROD2D) return run_marginal<GaussianProductKernel2d<double>>(r, dim_idx);
    if (kind == EPAN_PROD2D) return run_marginal<EpanechnikovProductKernel2d<double>>(r, dim_idx);
    return 5;
  } catch (const std::invalid_argument &) { return 2; }
  catch (...) { return 9; }
}

// Kernel normalisation C(h) exactly as the reference computes it, including the
// float-typed bandwidth of GaussianTraits<1,double>::normalization
// (include/Kernels/KernelTraits.h:143).
double ref_kde_normalization(int kind, int dim, const double *h) {
  if (dim == 1) {
    switch (kind) {
      case GAUSS: return GaussianKernel<1, double>(h[0]).normalization();
      case EPAN: return EpanechnikovKernel<1, double>(h[0]).normalization();
      case GAUSS_CONV1D: return GaussianConvKernel1d<double>(h[0]).normalization();
      case EPAN_CONV1D: return EpanechnikovConvKernel1d<double>(h[0]).normalization();
    }
  } else {
    switch (kind) {
      case GAUSS: return GaussianKernel<2, double>(h[0]).normalization();
      case EPAN: return EpanechnikovKernel<2, double>(h[0]).normalization();
      case GAUSS_PROD2D: return GaussianProductKernel2d<double>(h[0], h[1]).normalization();
      case EPAN_PROD2D: return EpanechnikovProductKernel2d<double>(h[0], h[1]).normalization();
      case GAUSS_PROD_CONV2D: return GaussianProductConvKernel2d<double>(h[0], h[1]).normalization();
      case EPAN_PROD_CONV2D: return EpanechnikovProductConvKernel2d<double>(h[0], h[1]).normalization();
    }
  }
  return 0.0;
}

}  // extern "C"
