// Drop-in test: reference-style C++ code compiled with g++ against the bbrcit
// names of include/bbkde/ and linked with libbbkde.so.
//
// Like the reference's CPU-vs-GPU checks (test/test_cukde0.cc:46-105,
// test/test_cukde2.cc:42-97), each case computes the density with a plain FP64
// CPU loop over the kernels' host unnormalized_eval and compares it with the GPU
// class using approximately_equal(rel 1e-6, abs 1e-8). Prints PASSED / FAILED per
// case; exits non-zero if any case fails.
#include <cmath>
#include <cstdio>
#include <iostream>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include <CudaDirectKde.h>
#include <FloatUtils.h>
#include <KernelDensity.h>
#include <Kernels/EpanechnikovKernel.h>
#include <Kernels/EpanechnikovProductKernel2d.h>
#include <Kernels/GaussianKernel.h>
#include <Kernels/GaussianProductKernel2d.h>

using namespace bbrcit;

namespace {

int failures = 0;

void report(const std::string &name, bool ok, const std::string &detail = "") {
  std::cout << (ok ? "PASSED " : "FAILED ") << name;
  if (!detail.empty()) std::cout << " (" << detail << ")";
  std::cout << std::endl;
  if (!ok) ++failures;
}

template <typename PointT>
void bimodal(std::mt19937 &e, std::vector<PointT> &pts, int n, bool weighted) {
  std::normal_distribution<double> g(0.0, 1.0);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  pts.clear();
  for (int i = 0; i < n; ++i) {
    bool first = u(e) < 0.5;
    double x = (double)(float)(g(e) * 0.5 + (first ? -1.0 : 1.0));
    double y = (double)(float)(g(e) * 0.5 + (first ? -1.0 : 1.0));
    double w = weighted ? 0.5 + u(e) : 1.0;
    pts.push_back({{x, y}, {w}});
  }
}

template <typename PointT>
void grid(std::vector<PointT> &pts, double lo, double hi, int steps) {
  pts.clear();
  double d = (hi - lo) / steps;
  for (int j = 0; j < steps; ++j)
    for (int i = 0; i < steps; ++i)
      pts.push_back({{(double)(float)(lo + i * d), (double)(float)(lo + j * d)}});
}

// FP64 CPU density at q over data points with their mass / abw attributes.
template <typename K, typename Pts, typename Q>
double cpu_density(const K &k, const Pts &data, const Q &q, bool normalized = true) {
  double s = 0;
  for (const auto &d : data)
    s += double(d.attributes().mass()) *
         double(k.unnormalized_eval(q.point(), d.point(), d.attributes().abw()));
  return normalized ? s * double(k.normalization()) : s;
}

template <typename V1, typename V2>
bool consistent(const V1 &cpu, const V2 &gpu, size_t n, std::string &why) {
  for (size_t i = 0; i < n; ++i) {
    if (!approximately_equal(double(cpu[i]), double(gpu[i]), 1e-6, 1e-8)) {
      why = "i=" + std::to_string(i) + " cpu=" + std::to_string(cpu[i]) +
            " gpu=" + std::to_string(gpu[i]);
      return false;
    }
  }
  return true;
}

using Attr = AdaKdeAttributes<double>;
using Pt = DecoratedPoint<2, Attr, double>;

void test_cuda_direct_kde() {
  // test_cukde0.cc: Epanechnikov 2-D, 4096 x 4096 points, bandwidth 1.
  std::mt19937 e(11);
  std::vector<Pt> refs, queries;
  bimodal(e, refs, 4096, false);
  bimodal(e, queries, 4096, false);
  for (auto &p : refs) p.attributes().set_mass(1.0 / 4096);
  CudaDirectKde<2, float, EpanechnikovKernel<2, float>> cu(refs, queries);
  cu.kernel().set_bandwidth(1.0f);
  std::vector<float> gpu;
  cu.eval(0, refs.size() - 1, 0, queries.size() - 1, gpu);
  std::vector<double> cpu(queries.size());
  EpanechnikovKernel<2, double> k(1.0);
  for (size_t i = 0; i < queries.size(); ++i) cpu[i] = cpu_density(k, refs, queries[i]);
  std::string why;
  report("CudaDirectKde::eval full range", consistent(cpu, gpu, cpu.size(), why), why);

  // test_cukde2.cc: closed sub-ranges, result[k - q_i].
  std::vector<Pt> half(refs.begin() + 1000, refs.begin() + 3001);
  cu.unnormalized_eval(1000, 3000, 512, 1535, gpu);
  bool ok = gpu.size() >= 1024;
  for (size_t i = 0; ok && i < 1024; ++i) {
    double c = cpu_density(k, half, queries[512 + i], false);
    if (!approximately_equal(c, double(gpu[i]), 1e-6, 1e-8 / 4096)) {
      ok = false;
      why = "i=" + std::to_string(i);
    }
  }
  report("CudaDirectKde::unnormalized_eval sub-range", ok, ok ? "" : why);

  bool threw = false;
  try { cu.eval(0, refs.size(), 0, 10, gpu); } catch (const std::out_of_range &) { threw = true; }
  report("CudaDirectKde out_of_range", threw);
  threw = false;
  try { cu.eval(10, 9, 0, 10, gpu); } catch (const std::invalid_argument &) { threw = true; }
  report("CudaDirectKde invalid_argument", threw);
}

void test_kernel_density() {
  using Kern = GaussianProductKernel2d<float>;
  using Kde = KernelDensity<2, Kern, double>;
  std::mt19937 e(7);
  std::vector<Pt> data, queries;
  bimodal(e, data, 3000, true);
  grid(queries, -3.0, 3.0, 60);
  Kde kde(data, 2);
  kde.kernel().set_bandwidths(0.1f, 0.15f);

  // direct_eval (KernelDensityImpl.h:1196-1231)
  kde.direct_eval(queries);
  GaussianProductKernel2d<double> kd(0.1f, 0.15f);   // the float kernel's bandwidths
  std::vector<double> cpu(queries.size()), gpu(queries.size());
  for (size_t i = 0; i < queries.size(); ++i) {
    cpu[i] = cpu_density(kd, kde.points(), queries[i]);
    gpu[i] = queries[i].attributes().value();
  }
  std::string why;
  report("KernelDensity::direct_eval", consistent(cpu, gpu, cpu.size(), why), why);

  Pt one{{0.5, -0.25}};
  double v = kde.direct_eval(one);
  report("KernelDensity::direct_eval(point)",
         approximately_equal(v, cpu_density(kd, kde.points(), one), 1e-6, 1e-8));

  // adapt_density (KernelDensityImpl.h:291-359): check the local bandwidths
  // against an FP64 CPU pilot pass.
  kde.kernel().set_bandwidths(0.05f, 0.05f);
  kde.adapt_density(0.5, 0.0, 0.0);   // rel_err = abs_err = 0: the exact pilot
  const auto &pts = kde.points();
  GaussianProductKernel2d<double> kp(0.05f, 0.05f);
  double logg = 0;
  std::vector<double> pilot(pts.size());
  for (size_t i = 0; i < pts.size(); ++i) {
    double s = 0;
    for (const auto &d : pts)
      s += double(d.attributes().weight()) * kp.unnormalized_eval(pts[i].point(), d.point());
    pilot[i] = s * kp.normalization();
    logg += double(pts[i].attributes().weight()) * std::log(pilot[i]);
  }
  double g = std::exp(logg);
  bool ok = true;
  for (size_t i = 0; i < pts.size() && ok; ++i) {
    double bw = std::pow(pilot[i] / g, -0.5);
    ok = approximately_equal(bw, double(pts[i].attributes().abw()), 2e-6, 0.0) &&
         approximately_equal(double(pts[i].attributes().weight()) / (bw * bw),
                             double(pts[i].attributes().mass()), 4e-6, 0.0);
    if (!ok) why = "i=" + std::to_string(i);
  }
  report("KernelDensity::adapt_density", ok, ok ? "" : why);

  // The reference's default tolerances (rel 1e-6, abs 1e-6): every pilot value
  // within max(1e-6 f, 1e-6) / 2 of the exact one (plus FP32 rounding), so the
  // bandwidth factor (f / g)^-1/2 moves by at most half that relative change
  // and half the relative change of g.
  std::vector<double> abw_exact(pts.size());
  for (size_t i = 0; i < pts.size(); ++i) abw_exact[i] = double(pts[i].attributes().abw());
  kde.adapt_density(0.5);
  ok = true;
  for (size_t i = 0; i < pts.size() && ok; ++i) {
    const double rel_pilot = 0.5e-6 * std::max(1.0, 1.0 / pilot[i]) + 2e-7;
    ok = approximately_equal(abw_exact[i], double(pts[i].attributes().abw()),
                             rel_pilot + 1e-6, 0.0);
    if (!ok) why = "i=" + std::to_string(i);
  }
  report("KernelDensity::adapt_density (rel 1e-6, abs 1e-6)", ok, ok ? "" : why);
  kde.adapt_density(0.5, 0.0, 0.0);

  // adaptive direct_eval uses the adapted attributes
  kde.direct_eval(queries);
  for (size_t i = 0; i < queries.size(); ++i) {
    cpu[i] = cpu_density(kp, kde.points(), queries[i]);
    gpu[i] = queries[i].attributes().value();
  }
  report("KernelDensity adaptive direct_eval", consistent(cpu, gpu, cpu.size(), why), why);

  bool threw = false;
  try { kde.adapt_density(1.5); } catch (const std::invalid_argument &) { threw = true; }
  report("adapt_density invalid_argument", threw);
}

void test_cross_validation() {
  using Kern = EpanechnikovProductKernel2d<double>;
  using Kde = KernelDensity<2, Kern, double>;
  std::mt19937 e(3);
  std::vector<Pt> data;
  bimodal(e, data, 2500, true);
  Kde kde(data);
  kde.kernel().set_bandwidths(0.4, 0.3);
  const auto &pts = kde.points();
  Kern k(0.4, 0.3);
  EpanechnikovProductConvKernel2d<double> kc(0.4, 0.3);
  double lik = 0, llo = 0, sq = 0;
  for (size_t i = 0; i < pts.size(); ++i) {
    double f = 0, fc = 0;
    for (size_t j = 0; j < pts.size(); ++j) {
      fc += pts[j].attributes().mass() * kc.unnormalized_eval(pts[i].point(), pts[j].point());
      if (j != i)
        f += pts[j].attributes().mass() * k.unnormalized_eval(pts[i].point(), pts[j].point());
    }
    f *= k.normalization();
    fc *= kc.normalization();
    lik += pts[i].attributes().weight() * std::log(f);
    llo += pts[i].attributes().weight() * f;
    sq += pts[i].attributes().weight() * fc;
  }
  double gl = kde.likelihood_cross_validate();
  double gs = kde.lsq_convolution_cross_validate();
  // An isolated point has leave-one-out density 0 under the compact-support
  // kernel, so both scores may be -inf (the reference's log(0) as well).
  bool same_inf = std::isinf(gl) && std::isinf(lik) && (gl < 0) == (lik < 0);
  report("likelihood_cross_validate", same_inf || approximately_equal(gl, lik, 1e-9, 0.0),
         std::to_string(gl) + " vs " + std::to_string(lik));
  report("lsq_convolution_cross_validate", approximately_equal(gs, sq - 2 * llo, 1e-9, 0.0),
         std::to_string(gs) + " vs " + std::to_string(sq - 2 * llo));
  // test_kde20.cc compares the convolution and numerical-integration forms.
  double gn = lsq_numint_cross_validate(kde, -4.0, 4.0, 400, -4.0, 4.0, 400);
  report("lsq_numint_cross_validate ~ lsq_convolution", std::fabs(gn - gs) < 2e-3 * std::fabs(gs),
         std::to_string(gn) + " vs " + std::to_string(gs));
}

void test_gaussian_likelihood() {
  using Kern = GaussianProductKernel2d<float>;
  std::mt19937 e(9);
  std::vector<Pt> data;
  bimodal(e, data, 2000, true);
  KernelDensity<2, Kern, double> kde(data);
  kde.kernel().set_bandwidths(0.12f, 0.2f);
  const auto &pts = kde.points();
  GaussianProductKernel2d<double> k(0.12f, 0.2f);
  double lik = 0;
  for (size_t i = 0; i < pts.size(); ++i) {
    double f = 0;
    for (size_t j = 0; j < pts.size(); ++j)
      if (j != i) f += pts[j].attributes().mass() * k.unnormalized_eval(pts[i].point(), pts[j].point());
    lik += pts[i].attributes().weight() * std::log(f * k.normalization());
  }
  double gl = kde.likelihood_cross_validate(0.0, 0.0);   // exact sums
  report("likelihood_cross_validate (Gaussian, FP32C)", approximately_equal(gl, lik, 1e-6, 0.0),
         std::to_string(gl) + " vs " + std::to_string(lik));
  // Default tolerances (rel 1e-6, abs 1e-6): each leave-one-out density within
  // max(1e-6 f, 1e-6) / 2, so each log term within that over f.
  double bound = 0;
  for (size_t i = 0; i < pts.size(); ++i) {
    double f = 0;
    for (size_t j = 0; j < pts.size(); ++j)
      if (j != i) f += pts[j].attributes().mass() * k.unnormalized_eval(pts[i].point(), pts[j].point());
    f *= k.normalization();
    bound += pts[i].attributes().weight() * (0.5e-6 * std::max(f, 1.0) + 2e-7 * f) / f;
  }
  double gt = kde.likelihood_cross_validate();
  report("likelihood_cross_validate (rel 1e-6, abs 1e-6)", std::fabs(gt - lik) <= bound,
         std::to_string(gt) + " vs " + std::to_string(lik) + " bound " + std::to_string(bound));
}

void test_one_dimensional() {
  using P1 = DecoratedPoint<1, Attr, double>;
  std::mt19937 e(5);
  std::normal_distribution<double> g(0.0, 1.0);
  std::vector<P1> data, queries;
  for (int i = 0; i < 5000; ++i) data.push_back({{(double)(float)g(e)}, {1.0}});
  for (int i = 0; i < 2000; ++i) queries.push_back({{(double)(float)(-4.0 + i * 0.004)}});
  KernelDensity<1, GaussianKernel<1, float>, double> kde(data);
  kde.kernel().set_bandwidth(0.02f);
  kde.direct_eval(queries);
  GaussianKernel<1, double> k(0.02f);
  std::vector<double> cpu(queries.size()), gpu(queries.size());
  for (size_t i = 0; i < queries.size(); ++i) {
    cpu[i] = cpu_density(k, kde.points(), queries[i]);
    gpu[i] = queries[i].attributes().value();
  }
  std::string why;
  report("1-D GaussianKernel direct_eval", consistent(cpu, gpu, cpu.size(), why), why);
}

}  // namespace

void test_tolerance_eval_and_device_numint() {
  // KernelDensity::eval(queries, rel_err, abs_err) with an FP32 kernel runs the
  // culled sum (every value within rel_err of the full sum); the reference's
  // tree eval promises the same tolerance.
  using Kern = GaussianKernel<2, float>;
  std::mt19937 e(21);
  std::vector<Pt> data, queries;
  bimodal(e, data, 6000, true);
  grid(queries, -3.0, 3.0, 120);
  KernelDensity<2, Kern, double> kde(data);
  kde.kernel().set_bandwidth(0.08f);
  kde.adapt_density(0.5);
  std::vector<Pt> got(queries);
  kde.eval(got, 1e-6, 1e-8);
  GaussianKernel<2, double> k(0.08f);
  std::vector<double> cpu(queries.size()), gpu(queries.size());
  for (size_t i = 0; i < queries.size(); ++i) {
    cpu[i] = cpu_density(k, kde.points(), queries[i]);
    gpu[i] = got[i].attributes().value();
  }
  std::string why;
  report("KernelDensity::eval(rel 1e-6) culled", consistent(cpu, gpu, cpu.size(), why), why);

  // lsq_numint_cross_validate on the device (FP32 kernel) against the host sum
  // of the same terms over FP64 CPU densities.
  const double x0 = -4, x1 = 4, y0 = -4, y1 = 4;
  const int sx = 160, sy = 160;
  double dev = lsq_numint_cross_validate(kde, x0, x1, sx, y0, y1, sy);
  const auto &pts = kde.points();
  double llo = 0, sq = 0;
  for (size_t i = 0; i < pts.size(); ++i) {
    double f = 0;
    for (size_t j = 0; j < pts.size(); ++j)
      if (j != i)
        f += pts[j].attributes().mass() *
             k.unnormalized_eval(pts[i].point(), pts[j].point(), pts[j].attributes().abw());
    llo += pts[i].attributes().weight() * f * k.normalization();
  }
  const double dx = (x1 - x0) / sx, dy = (y1 - y0) / sy;
  for (int j = 0; j < sy; ++j)
    for (int i = 0; i < sx; ++i) {
      Pt q = {{(double)(float)(x0 + i * dx), (double)(float)(y0 + j * dy)}};
      double f = cpu_density(k, pts, q);
      sq += f * f * dx * dy;
    }
  double want = sq - 2 * llo;
  report("lsq_numint_cross_validate on the device", std::fabs(dev - want) < 2e-6 * std::fabs(want),
         std::to_string(dev) + " vs " + std::to_string(want));
}

int main() {
  try {
    test_cuda_direct_kde();
    test_kernel_density();
    test_cross_validation();
    test_gaussian_likelihood();
    test_one_dimensional();
    test_tolerance_eval_and_device_numint();
  } catch (const std::exception &ex) {
    std::cout << "ERROR " << ex.what() << std::endl;
    return 2;
  }
  std::cout << (failures ? "SOME TESTS FAILED" : "ALL PASSED") << std::endl;
  return failures ? 1 : 0;
}
