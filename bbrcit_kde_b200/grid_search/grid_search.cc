// grid_search -- bandwidth selection for weighted 2-D data by least-squares cross
// validation, then density evaluation on a plotting grid.
//
// The same command line, configuration keys, steps and output files as the
// reference's driver (grid_search/grid_search.cc:158-552, grid_search/cv_utils*.h,
// grid_search/template.cfg), written over the C ABI of libbbkde.so and without
// Boost:
//   grid_search [--key=value ...] config_fname
// Keys given on the command line take precedence over the configuration file
// (as boost::program_options stores the command line first).
//
// What changes on the B200: the reference scores the bandwidth grid one
// bandwidth at a time, each a full self-evaluation (grid_search.cc:370-402).
// Here the convolution-form LSQ CV of the whole grid (up to 64 x 64 strictly
// increasing bandwidths) is one bbkde_cv_batch launch; the numerical-integration
// form and the adaptive case run bbkde_lsq_numint_cv per bandwidth. Densities on
// the plotting grid use the culled sum with the configured relative tolerance
// (bbkde_eval_culled) and the adaptive pilots a culled self-sum to that tolerance
// (bbkde_adapt_density_tol), where the reference uses its tree evaluation with
// the same tolerance. The Kd-tree leaf sizes and the GPU block size are accepted
// and not needed.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/bbkde.h"

namespace {

using Clock = std::chrono::high_resolution_clock;

double ms_since(Clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

std::string trim(const std::string &s) {
  const char *ws = " \t\r\n";
  const size_t b = s.find_first_not_of(ws);
  if (b == std::string::npos) return "";
  return s.substr(b, s.find_last_not_of(ws) - b + 1);
}

// Options: "key = value" lines of the configuration file ('#' starts a comment),
// overridden by --key=value / --key value on the command line.
class Options {
 public:
  void set_if_absent(const std::string &k, const std::string &v) {
    if (!vals_.count(k)) vals_[k] = v;
  }
  void read_file(const std::string &path) {
    std::ifstream fin(path);
    if (!fin) throw std::runtime_error("cannot open config file: " + path);
    std::string line;
    while (std::getline(fin, line)) {
      const size_t hash = line.find('#');
      if (hash != std::string::npos) line = line.substr(0, hash);
      line = trim(line);
      if (line.empty()) continue;
      const size_t eq = line.find('=');
      if (eq == std::string::npos) throw std::runtime_error("malformed config line: " + line);
      set_if_absent(trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
    }
  }
  const std::string &str(const std::string &k) const {
    auto it = vals_.find(k);
    if (it == vals_.end()) throw std::runtime_error("missing option '" + k + "'");
    return it->second;
  }
  double real(const std::string &k) const { return std::stod(str(k)); }
  int integer(const std::string &k) const { return std::stoi(str(k)); }
  bool flag(const std::string &k) const {
    const std::string v = str(k);
    if (v == "true" || v == "1" || v == "yes" || v == "on") return true;
    if (v == "false" || v == "0" || v == "no" || v == "off") return false;
    throw std::runtime_error("option '" + k + "' is not a boolean: " + v);
  }

 private:
  std::map<std::string, std::string> vals_;
};

std::vector<double> numbers(const std::string &s) {
  std::istringstream is(s);
  std::vector<double> v;
  double x;
  while (is >> x) v.push_back(x);
  return v;
}

void check(int rc, bbkde_ctx *ctx) {
  if (rc == BBKDE_OK) return;
  throw std::runtime_error(ctx ? bbkde_ctx_last_error(ctx) : bbkde_status_string(rc));
}

// Regular grid with both end points (cv_utils_impl.h: generate_2dgrid), y outer.
std::vector<std::pair<double, double>> grid_points(double x0, double x1, int sx, double y0,
                                                   double y1, int sy) {
  std::vector<std::pair<double, double>> g;
  const double dx = (x1 - x0) / sx, dy = (y1 - y0) / sy;
  for (int j = 0; j <= sy; ++j)
    for (int i = 0; i <= sx; ++i) g.emplace_back(x0 + i * dx, y0 + j * dy);
  return g;
}

// cv_utils.cpp: write_2dgrid_values -- the x ticks, the y ticks, then one row of
// steps_x + 1 values per y.
void write_grid_values(const std::string &path, const std::vector<double> &v, double x0,
                       double x1, int sx, double y0, double y1, int sy) {
  std::ofstream os(path);
  if (!os) throw std::runtime_error("cannot write " + path);
  const double dx = (x1 - x0) / sx, dy = (y1 - y0) / sy;
  for (int i = 0; i <= sx; ++i) os << x0 + i * dx << " ";
  os << std::endl;
  for (int i = 0; i <= sy; ++i) os << y0 + i * dy << " ";
  os << std::endl;
  for (size_t i = 0; i < v.size(); ++i) {
    if (i % (size_t)(sx + 1) == 0 && i) os << std::endl;
    os << v[i] << " ";
  }
  os << std::endl;
}

bool strictly_increasing_positive(const std::vector<double> &v) {
  for (size_t i = 0; i < v.size(); ++i)
    if (!(v[i] > 0) || (i && !(v[i] > v[i - 1]))) return false;
  return !v.empty();
}

struct Session {
  bbkde_ctx *ctx = nullptr;
  std::vector<double> xy, w;   // reference points (AoS) and raw weights
  ~Session() { bbkde_ctx_destroy(ctx); }

  bbkde_kernel_desc kernel(double bx, double by) const {
    bbkde_kernel_desc k;
    k.kind = BBKDE_EPANECHNIKOV_PRODUCT_2D;
    k.dim = 2;
    k.h[0] = bx;
    k.h[1] = by;
    k.flags = 0;
    k.reserved = 0;
    return k;
  }
  // Adaptive densities as the reference's adapt_density(alpha, rel_tol, abs_tol)
  // (grid_search.cc:266-268, :508-510): the pilot to max(rel_tol f, abs_tol) when
  // rel_tol lies in [0, 1) and a tolerance is set, else the exact pilot.
  void adapt(const bbkde_kernel_desc &k, double alpha, double rel_tol, double abs_tol) {
    if (rel_tol >= 0 && rel_tol < 1 && abs_tol >= 0 && (rel_tol > 0 || abs_tol > 0))
      check(bbkde_adapt_density_tol(ctx, &k, alpha, rel_tol, abs_tol, nullptr, nullptr, nullptr,
                                    nullptr),
            ctx);
    else
      check(bbkde_adapt_density(ctx, &k, alpha, BBKDE_FP32C, nullptr, nullptr, nullptr, nullptr),
            ctx);
  }
  // Density at the grid points (x0..x1 by sx, y0..y1 by sy, ends included).
  std::vector<double> eval_grid(double bx, double by, double x0, double x1, int sx, double y0,
                                double y1, int sy, double rel_tol, double abs_tol) {
    auto g = grid_points(x0, x1, sx, y0, y1, sy);
    std::vector<double> q(2 * g.size()), out(g.size());
    for (size_t i = 0; i < g.size(); ++i) {
      q[2 * i] = g[i].first;
      q[2 * i + 1] = g[i].second;
    }
    check(bbkde_upload(ctx, BBKDE_QUERY, 2, (int64_t)g.size(), q.data(), nullptr, nullptr,
                       nullptr),
          ctx);
    const bbkde_kernel_desc k = kernel(bx, by);
    if (rel_tol >= 0 && rel_tol < 1 && abs_tol >= 0 && (rel_tol > 0 || abs_tol > 0)) {
      check(bbkde_eval_tol(ctx, &k, 1, rel_tol, abs_tol, out.data(), 0, nullptr), ctx);
    } else {
      const int64_t n = bbkde_size(ctx, BBKDE_REFERENCE);
      check(bbkde_eval_range(ctx, &k, 0, n - 1, 0, (int64_t)g.size() - 1, 1, BBKDE_FP32C,
                             out.data(), 0),
            ctx);
    }
    return out;
  }
};

void usage() {
  std::cout << "\nUsage: grid_search [--key=value ...] config_fname\n\n"
               "Reads weighted 2-D points (x y w per line), selects (hx, hy) of the\n"
               "Epanechnikov product kernel by least-squares cross validation over a\n"
               "bandwidth grid, and writes the density on a plotting grid, as configured\n"
               "by the keys of the configuration file (see grid_search/example.cfg).\n"
            << std::endl;
}

void run(const Options &o) {
  const double rel_tol = o.real("rel_tol"), abs_tol = o.real("abs_tol");
  std::cout << "+ performance parameters: \n\n";
  std::cout << "  relative tolerance: " << rel_tol << "\n";
  std::cout << "  absolute tolerance: " << abs_tol << "\n\n";
  const int device = o.integer("cuda_device_number");
  (void)o.integer("gpu_block_size");
  (void)o.integer("refpt_max_leaf_size");
  (void)o.integer("qgrid_max_leaf_size");

  Session s;
  check(bbkde_ctx_create(device, &s.ctx), nullptr);
  int sms = 0;
  bbkde_device_info(s.ctx, &sms, nullptr);
  std::cout << "  gpu device number used for this session: " << device << " (" << sms
            << " SMs)\n\n";

  // 1. reference data (cv_utils_impl.h: read_2dpoints; write_2dscatter_data)
  const std::string in = o.str("input_refpts_fname");
  std::cout << "+ reading in reference data. \n\n";
  {
    std::ifstream fin(in);
    if (!fin) throw std::runtime_error("cannot open file " + in + ". ");
    double x, y, w;
    while (fin >> x >> y >> w) {
      s.xy.push_back(x);
      s.xy.push_back(y);
      s.w.push_back(w);
    }
  }
  const int64_t n = (int64_t)s.w.size();
  std::cout << "  => found " << n << " points. \n\n";
  {
    const std::string out = o.str("output_scatter_fname");
    std::ofstream fout(out);
    for (int64_t i = 0; i < n; ++i) fout << s.xy[2 * i] << " " << s.xy[2 * i + 1] << std::endl;
    std::cout << "  => wrote results to: " << out << ". \n\n";
  }

  // 2. the estimator: weights normalised to sum 1, masses = weights
  //    (KernelDensityImpl.h:430-455), optionally adapted.
  const bool adaptive_cv = o.flag("use_adaptive_cv");
  const bool skip_cv = o.flag("skip_cross_validation");
  const double base_bwx = o.real("base_bwx"), base_bwy = o.real("base_bwy");
  const double alpha = o.real("alpha");
  double wsum = 0;
  for (double w : s.w) wsum += w;
  std::vector<double> wn(s.w.size());
  for (size_t i = 0; i < wn.size(); ++i) wn[i] = s.w[i] / wsum;
  std::cout << "+ constructing kernel density estimator. \n\n";
  std::cout << "  base bandwidth x: " << base_bwx << "\n  base bandwidth y: " << base_bwy
            << "\n\n";
  auto t0 = Clock::now();
  check(bbkde_upload(s.ctx, BBKDE_REFERENCE, 2, n, s.xy.data(), wn.data(), nullptr, wn.data()),
        s.ctx);
  std::cout << "  => running time: " << ms_since(t0) << " ms. \n\n";
  std::cout << "  perform adaptive density cross validation: "
            << (adaptive_cv ? "true" : "false") << "\n";
  std::cout << "  skip cross validation: " << (skip_cv ? "true" : "false") << "\n\n";
  if (adaptive_cv && !skip_cv) {
    std::cout << "  converting to adaptive density for cross validation. \n\n";
    std::cout << "  alpha: " << alpha << "\n\n";
    const bbkde_kernel_desc k = s.kernel(base_bwx, base_bwy);
    t0 = Clock::now();
    s.adapt(k, alpha, rel_tol, abs_tol);
    std::cout << "  => running time: " << ms_since(t0) << " ms. \n\n";
  }

  // 3. grid search
  const bool manual = o.flag("use_manual_bwgrid");
  std::string method = o.str("cv_method");
  const double sbx = o.real("start_bwx"), ebx = o.real("end_bwx");
  const double sby = o.real("start_bwy"), eby = o.real("end_bwy");
  const int nbx = o.integer("steps_bwx"), nby = o.integer("steps_bwy");
  const double sqix = o.real("start_qix"), eqix = o.real("end_qix");
  const double sqiy = o.real("start_qiy"), eqiy = o.real("end_qiy");
  const int nqix = o.integer("steps_qix"), nqiy = o.integer("steps_qiy");
  double best_bwx = base_bwx, best_bwy = base_bwy;
  if (!skip_cv) {
    if (adaptive_cv) method = "lsq_numint";   // grid_search.cc:296-298
    if (method != "lsq_conv" && method != "lsq_numint")
      throw std::invalid_argument("grid_search: unrecognized cv method. ");
    // bandwidth lists: x values and y values of the crossed grid
    std::vector<double> hx, hy;
    std::vector<std::pair<double, double>> pairs;
    if (!manual) {
      for (int i = 0; i <= nbx; ++i) hx.push_back(sbx + i * ((ebx - sbx) / nbx));
      for (int j = 0; j <= nby; ++j) hy.push_back(sby + j * ((eby - sby) / nby));
      pairs = grid_points(sbx, ebx, nbx, sby, eby, nby);      // y outer, x inner
    } else {
      hx = numbers(o.str("manual_bwx"));
      hy = numbers(o.str("manual_bwy"));
      for (double a : hx)
        for (double b : hy) pairs.emplace_back(a, b);         // x outer, y inner
    }
    if (method == "lsq_conv")
      std::cout << "+ using convolution based least squares cross validation. \n\n";
    else
      std::cout << "+ using numerical integration based least squares cross validation. \n"
                << "    grid dimensions: " << nqix << " by " << nqiy << "\n\n";
    std::cout << "  grid searching over " << pairs.size() << " bandwidths: \n\n";

    std::vector<double> scores(pairs.size());
    t0 = Clock::now();
    const bool batched = method == "lsq_conv" && !adaptive_cv && hx.size() <= 64 &&
                         hy.size() <= 64 && strictly_increasing_positive(hx) &&
                         strictly_increasing_positive(hy);
    if (batched) {
      // every (hx, hy) in one launch; lsq[a * |hy| + b] belongs to (hx[a], hy[b])
      bbkde_dataset set = {n, s.xy.data(), s.w.data()};
      std::vector<double> lik(hx.size() * hy.size()), lsq(lik.size());
      check(bbkde_cv_batch(s.ctx, BBKDE_EPANECHNIKOV_PRODUCT_2D, 1, &set, (int)hx.size(),
                           hx.data(), (int)hy.size(), hy.data(), BBKDE_FP64, lik.data(),
                           lsq.data()),
            s.ctx);
      for (size_t p = 0; p < pairs.size(); ++p) {
        const size_t a = manual ? p / hy.size() : p % hx.size();
        const size_t b = manual ? p % hy.size() : p / hx.size();
        scores[p] = lsq[a * hy.size() + b];
      }
    } else {
      for (size_t p = 0; p < pairs.size(); ++p) {
        const bbkde_kernel_desc k = s.kernel(pairs[p].first, pairs[p].second);
        if (method == "lsq_conv") {
          check(bbkde_lsq_conv_cv(s.ctx, &k, BBKDE_FP32C, &scores[p]), s.ctx);
        } else {
          // grid of lsq_numint_cross_validate: end points excluded (KernelDensityImpl.h:69-75)
          bbkde_grid g = {nqix, nqiy, sqix, eqix, sqiy, eqiy};
          check(bbkde_lsq_numint_cv(s.ctx, &k, &g, BBKDE_FP32C, &scores[p]), s.ctx);
        }
      }
    }
    const double elapsed = ms_since(t0);
    double best_cv = std::numeric_limits<double>::max();
    for (size_t p = 0; p < pairs.size(); ++p) {
      if (scores[p] < best_cv) {
        best_cv = scores[p];
        best_bwx = pairs[p].first;
        best_bwy = pairs[p].second;
      }
      std::cout << "  (" << pairs[p].first << ", " << pairs[p].second << ") " << scores[p]
                << "\n";
    }
    std::cout << "\n  => best bandwidth: (" << best_bwx << ", " << best_bwy
              << "), cv score = " << best_cv << "\n\n";
    std::cout << "  => running time per iteration: " << elapsed / pairs.size() << " ms  ("
              << (batched ? "one batched launch" : "one bandwidth at a time") << ")\n\n";
    if (!manual) {
      const std::string out = o.str("output_gridsearch_fname");
      write_grid_values(out, scores, sbx, ebx, nbx, sby, eby, nby);
      std::cout << "  => wrote results to: " << out << ". \n\n";
    }
  }

  // 4. the non-adapted density on the plotting grid
  bool use_best = o.flag("use_gridsearch_best");
  if (skip_cv) use_best = false;
  const double sqx = o.real("start_qx"), eqx = o.real("end_qx");
  const double sqy = o.real("start_qy"), eqy = o.real("end_qy");
  const int nqx = o.integer("steps_qx"), nqy = o.integer("steps_qy");
  check(bbkde_unadapt_density(s.ctx), s.ctx);
  const double bx = (use_best && !adaptive_cv) ? best_bwx : base_bwx;
  const double by = (use_best && !adaptive_cv) ? best_bwy : base_bwy;
  std::cout << "+ evaluating cross validated non-adapted kernel density over plotting grid. \n\n";
  std::cout << "  grid dimensions: " << nqx << "x" << nqy << "\n  x bandwidth: " << bx
            << "\n  y bandwidth: " << by << "\n\n";
  t0 = Clock::now();
  std::vector<double> dens = s.eval_grid(bx, by, sqx, eqx, nqx, sqy, eqy, nqy, rel_tol, abs_tol);
  std::cout << "  => running time: " << ms_since(t0) << " ms. \n\n";
  {
    const std::string out = o.str("output_eval_fname");
    write_grid_values(out, dens, sqx, eqx, nqx, sqy, eqy, nqy);
    std::cout << "  => wrote results to: " << out << ". \n\n";
  }

  // 5. the adaptive density on the plotting grid
  const double before_bwx = (!adaptive_cv && use_best) ? best_bwx : base_bwx;
  const double before_bwy = (!adaptive_cv && use_best) ? best_bwy : base_bwy;
  std::cout << "+ converting to adaptive density for evaluation. \n\n";
  std::cout << "  base bandwidth x: " << before_bwx << "\n  base bandwidth y: " << before_bwy
            << "\n  alpha: " << alpha << "\n\n";
  const bbkde_kernel_desc kb = s.kernel(before_bwx, before_bwy);
  t0 = Clock::now();
  s.adapt(kb, alpha, rel_tol, abs_tol);
  std::cout << "  => running time: " << ms_since(t0) << " ms. \n\n";
  double after_bwx = before_bwx, after_bwy = before_bwy;
  if (adaptive_cv) {
    after_bwx = use_best ? best_bwx : o.real("adapted_base_bwx");
    after_bwy = use_best ? best_bwy : o.real("adapted_base_bwy");
  }
  std::cout << "+ evaluating cross validated adapted kernel density over plotting grid. \n\n";
  std::cout << "  final bandwidth x: " << after_bwx << "\n  final bandwidth y: " << after_bwy
            << "\n\n";
  t0 = Clock::now();
  dens = s.eval_grid(after_bwx, after_bwy, sqx, eqx, nqx, sqy, eqy, nqy, rel_tol, abs_tol);
  std::cout << "  => running time: " << ms_since(t0) << " ms. \n\n";
  const std::string out = o.str("output_adaptive_eval_fname");
  write_grid_values(out, dens, sqx, eqx, nqx, sqy, eqy, nqy);
  std::cout << "  => wrote results to: " << out << ". \n\n";
}

}  // namespace

int main(int argc, char **argv) {
  try {
    Options o;
    std::string config;
    for (int i = 1; i < argc; ++i) {
      const std::string a = argv[i];
      if (a == "--help" || a == "-h") {
        usage();
        return 0;
      }
      if (a.compare(0, 2, "--") == 0) {
        const size_t eq = a.find('=');
        if (eq != std::string::npos) {
          o.set_if_absent(a.substr(2, eq - 2), a.substr(eq + 1));
        } else if (i + 1 < argc) {
          o.set_if_absent(a.substr(2), argv[++i]);
        } else {
          throw std::runtime_error("option " + a + " needs a value");
        }
      } else {
        config = a;
      }
    }
    if (config.empty()) {
      usage();
      return 0;
    }
    o.read_file(config);
    run(o);
  } catch (const std::exception &e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
