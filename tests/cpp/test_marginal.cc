// Marginal densities through the C++ drop-in (MarginalDensityAssociator.h:22-128):
// the x and y marginals of a 2-D product-kernel density, evaluated on the device
// by direct_eval at 1-D queries.
//
//   test_marginal <in.bin> <out.bin>
//
// in.bin (little-endian): int64 n, int64 m, int64 kind (2 Gaussian product,
// 3 Epanechnikov product), int64 fp32 (1: float kernels, FP32-compensated device
// sums; 0: double kernels, FP64 device sums), double hx, hy, alpha (< 0: not
// adapted; else adapt_density(alpha, 0, 0), the exact pilot), then n rows
// (x, y, weight) and m query coordinates.
// out.bin: the x marginal at the m queries, the y marginal at the m queries, then
// for each marginal int64 k and k rows (coordinate, weight, mass, abw) of its points.
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <vector>

#include <KernelDensity.h>
#include <Kernels/EpanechnikovProductKernel2d.h>
#include <Kernels/GaussianProductKernel2d.h>
#include <MarginalDensityAssociator.h>

using namespace bbrcit;

namespace {

template <typename Kern>
int run(int64_t n, int64_t m, double hx, double hy, double alpha, const std::vector<double> &xyw,
        const std::vector<double> &q, FILE *out) {
  using Kde = KernelDensity<2, Kern, double>;
  using Assoc = MarginalDensityAssociator<Kde>;
  using P = typename Kde::DataPointType;
  using Real = typename Kern::FloatType;
  std::vector<P> pts;
  for (int64_t i = 0; i < n; ++i) {
    P p;
    p[0] = xyw[3 * i];
    p[1] = xyw[3 * i + 1];
    p.attributes() = AdaKdeAttributes<double>(xyw[3 * i + 2]);
    pts.push_back(p);
  }
  Kde kde(std::move(pts), 2);
  kde.kernel().set_bandwidths(Real(hx), Real(hy));
  if (alpha >= 0) kde.adapt_density(alpha, 0.0, 0.0);
  typename Assoc::MarginalDensityType mx = Assoc::marginal_density_x(kde);
  typename Assoc::MarginalDensityType my = Assoc::marginal_density_y(kde);
  for (auto *md : {&mx, &my}) {
    std::vector<typename Assoc::Point1d> qs(m);
    for (int64_t i = 0; i < m; ++i) qs[i][0] = q[i];
    md->direct_eval(qs);
    for (int64_t i = 0; i < m; ++i) {
      const double v = qs[i].attributes().value();
      std::fwrite(&v, sizeof v, 1, out);
    }
  }
  for (auto *md : {&mx, &my}) {
    const int64_t k = (int64_t)md->points().size();
    std::fwrite(&k, sizeof k, 1, out);
    for (const auto &p : md->points()) {
      const double row[4] = {p[0], p.attributes().weight(), p.attributes().mass(),
                             p.attributes().abw()};
      std::fwrite(row, sizeof(double), 4, out);
    }
  }
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::cerr << "usage: test_marginal <in.bin> <out.bin>\n";
    return 2;
  }
  FILE *in = std::fopen(argv[1], "rb");
  if (!in) return 3;
  int64_t hdr[4];
  double par[3];
  if (std::fread(hdr, sizeof(int64_t), 4, in) != 4 || std::fread(par, sizeof(double), 3, in) != 3)
    return 3;
  const int64_t n = hdr[0], m = hdr[1], kind = hdr[2], fp32 = hdr[3];
  std::vector<double> xyw(3 * n), q(m);
  if (std::fread(xyw.data(), sizeof(double), xyw.size(), in) != xyw.size() ||
      std::fread(q.data(), sizeof(double), q.size(), in) != q.size())
    return 3;
  std::fclose(in);
  FILE *out = std::fopen(argv[2], "wb");
  if (!out) return 3;
  int rc = 2;
  try {
    if (kind == 2 && fp32) rc = run<GaussianProductKernel2d<float>>(n, m, par[0], par[1], par[2], xyw, q, out);
    if (kind == 2 && !fp32) rc = run<GaussianProductKernel2d<double>>(n, m, par[0], par[1], par[2], xyw, q, out);
    if (kind == 3 && fp32) rc = run<EpanechnikovProductKernel2d<float>>(n, m, par[0], par[1], par[2], xyw, q, out);
    if (kind == 3 && !fp32) rc = run<EpanechnikovProductKernel2d<double>>(n, m, par[0], par[1], par[2], xyw, q, out);
  } catch (const std::exception &ex) {
    std::cerr << "ERROR " << ex.what() << "\n";
    rc = 4;
  }
  std::fclose(out);
  return rc;
}
