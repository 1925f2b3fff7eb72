// Sampling from a density through the C++ drop-in (KernelDensity::simulate,
// KernelDensityImpl.h:99-138): a weighted draw of a data point, then a draw from
// the kernel scaled by that point's adaptive bandwidth factor. Host code only;
// no device is needed.
//
//   test_simulate <kernel> <n_samples> <out.bin>
//
// kernel: gprod (GaussianProductKernel2d, hx 0.1, hy 0.2), gauss2 (GaussianKernel<2>,
// h 0.15), eprod (EpanechnikovProductKernel2d, 0.3, 0.2), epan2 (EpanechnikovKernel<2>,
// 0.25), epan1 (EpanechnikovKernel<1>, 0.2), gauss1 (GaussianKernel<1>, 0.1).
// Writes int64 n_points, int64 dim, the density's points in its own order as
// rows (coords..., weight, abw), then n_samples rows of coords, all doubles.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include <KernelDensity.h>
#include <Kernels/EpanechnikovKernel.h>
#include <Kernels/EpanechnikovProductKernel2d.h>
#include <Kernels/GaussianKernel.h>
#include <Kernels/GaussianProductKernel2d.h>

using namespace bbrcit;

namespace {

template <int D, typename Kern>
int run(const Kern &kern, long n_samples, const char *path) {
  using Kde = KernelDensity<D, Kern, double>;
  using P = typename Kde::DataPointType;
  // 1500 points of a two-component mixture with uneven weights and bandwidth
  // factors in [0.5, 2], set before construction (mass = w abw^-D as the
  // constructor computes it).
  std::mt19937 e(2024);
  std::normal_distribution<double> g(0.0, 1.0);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  std::vector<P> pts;
  for (int i = 0; i < 1500; ++i) {
    const bool first = u(e) < 0.3;
    P p;
    for (int d = 0; d < D; ++d) p[d] = (double)(float)(g(e) * 0.4 + (first ? -1.0 : 1.2));
    p.attributes() = AdaKdeAttributes<double>(0.2 + u(e));
    const double a = 0.5 + 1.5 * u(e);
    p.attributes().set_lower_abw(a);
    p.attributes().set_upper_abw(a);
    pts.push_back(p);
  }
  Kde kde(std::move(pts), 2);
  kde.kernel() = kern;
  FILE *f = std::fopen(path, "wb");
  if (!f) return 3;
  const int64_t np = (int64_t)kde.points().size(), dim = D;
  std::fwrite(&np, sizeof np, 1, f);
  std::fwrite(&dim, sizeof dim, 1, f);
  for (const auto &p : kde.points()) {
    double row[D + 2];
    for (int d = 0; d < D; ++d) row[d] = p[d];
    row[D] = p.attributes().weight();
    row[D + 1] = p.attributes().abw();
    std::fwrite(row, sizeof(double), D + 2, f);
  }
  std::mt19937_64 rng(77);
  std::vector<double> s;
  for (long i = 0; i < n_samples; ++i) {
    kde.simulate(rng, s);
    std::fwrite(s.data(), sizeof(double), D, f);
  }
  // the point-returning overload draws from the same distribution
  P q = kde.simulate(rng);
  (void)q;
  std::fclose(f);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 4) {
    std::cerr << "usage: test_simulate <kernel> <n_samples> <out.bin>\n";
    return 2;
  }
  const std::string k = argv[1];
  const long n = std::atol(argv[2]);
  if (k == "gprod") return run<2>(GaussianProductKernel2d<double>(0.1, 0.2), n, argv[3]);
  if (k == "gauss2") return run<2>(GaussianKernel<2, double>(0.15), n, argv[3]);
  if (k == "eprod") return run<2>(EpanechnikovProductKernel2d<double>(0.3, 0.2), n, argv[3]);
  if (k == "epan2") return run<2>(EpanechnikovKernel<2, double>(0.25), n, argv[3]);
  if (k == "epan1") return run<1>(EpanechnikovKernel<1, double>(0.2), n, argv[3]);
  if (k == "gauss1") return run<1>(GaussianKernel<1, double>(0.1), n, argv[3]);
  std::cerr << "unknown kernel " << k << "\n";
  return 2;
}
