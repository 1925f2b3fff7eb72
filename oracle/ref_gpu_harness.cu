// Test infrastructure, not product code: the reference's own GPU direct sum --
// CudaDirectKde<2, float, Kernel<float>>::unnormalized_eval and its eval_kernel
// (include/CudaDirectKde.h:126-215) -- compiled unmodified for sm_100a from the
// reference's headers (oracle/Makefile, target ref-gpu) into oracle/_ref/, behind a
// C ABI. It serves as a comparator on the same B200: oracle/ref_gpu_timing.py times
// it beside this project's pair sum, and the values are checked against the FP64
// oracle. Nothing in the product library links or calls this file.
//
// The call goes through the reference's public class exactly as its own tests do
// (test/test_cukde0.cc): host points are DecoratedPoint{{x, y}, AdaKdeAttributes}
// with mass and bandwidth factor set, the constructor copies them to the device as
// Point2d<float>, and unnormalized_eval launches eval_kernel with the given block
// size (one query per thread), allocating and copying the kernel object and the
// results synchronously on the legacy default stream, as the reference does.
#include <cstdint>
#include <random>  // the reference headers use std:: distributions without including it
#include <vector>

#include <cuda_runtime.h>

#include <Attributes/AdaKdeAttributes.h>
#include <CudaDirectKde.h>
#include <DecoratedPoint.h>
#include <Kernels/EpanechnikovKernel.h>
#include <Kernels/GaussianKernel.h>
#include <Kernels/GaussianProductKernel2d.h>

namespace {

using HostPoint = bbrcit::DecoratedPoint<2, bbrcit::AdaKdeAttributes<double>, double>;

std::vector<HostPoint> host_points(int64_t n, const double *xy, const double *mass,
                                   const double *abw) {
  std::vector<HostPoint> pts(n);
  for (int64_t i = 0; i < n; ++i) {
    pts[i][0] = xy[2 * i];
    pts[i][1] = xy[2 * i + 1];
    pts[i].attributes().set_mass(mass ? mass[i] : 1.0);
    const double a = abw ? abw[i] : 1.0;
    pts[i].attributes().set_lower_abw(a);
    pts[i].attributes().set_upper_abw(a);
  }
  return pts;
}

// reps timed calls after one untimed call; ms_per_call from CUDA events on the
// legacy default stream around the calls (each call is synchronous: kernel-object
// upload, launch, results download). out receives the normalised densities.
template <typename K>
int run(const K &kern, int64_t n, const double *xy, const double *mass, const double *abw,
        int64_t m, const double *q, int block, int reps, double *out, double *ms_per_call) {
  std::vector<HostPoint> refs = host_points(n, xy, mass, abw);
  std::vector<HostPoint> qs = host_points(m, q, nullptr, nullptr);
  bbrcit::CudaDirectKde<2, float, K> cu(refs, qs);
  cu.kernel() = kern;
  std::vector<float> res;
  cu.unnormalized_eval(0, (size_t)n - 1, 0, (size_t)m - 1, res, (size_t)block);
  if (cudaDeviceSynchronize() != cudaSuccess) return 3;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return 3;
  cudaEventRecord(e0, 0);
  for (int r = 0; r < reps; ++r)
    cu.unnormalized_eval(0, (size_t)n - 1, 0, (size_t)m - 1, res, (size_t)block);
  cudaEventRecord(e1, 0);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaGetLastError() != cudaSuccess) return 3;
  *ms_per_call = reps > 0 ? ms / reps : 0.0;
  const double c = kern.normalization();
  for (int64_t i = 0; i < m; ++i) out[i] = c * (double)res[i];
  return 0;
}

}  // namespace

extern "C" {

// kind numbered as in include/bbkde.h: 0 GaussianKernel<2, float> (h = hx),
// 1 EpanechnikovKernel<2, float> (h = hx), 2 GaussianProductKernel2d<float>.
// Returns 0, 2 for an unsupported kind or bad sizes, 3 for a CUDA error.
int ref_gpu_direct(int kind, double hx, double hy, int64_t n, const double *xy,
                   const double *mass, const double *abw, int64_t m, const double *q, int block,
                   int reps, double *out, double *ms_per_call) {
  if (n < 1 || m < 1 || block < 1 || block > 1024 || reps < 0) return 2;
  switch (kind) {
    case 0:
      return run(bbrcit::GaussianKernel<2, float>((float)hx), n, xy, mass, abw, m, q, block,
                 reps, out, ms_per_call);
    case 1:
      return run(bbrcit::EpanechnikovKernel<2, float>((float)hx), n, xy, mass, abw, m, q, block,
                 reps, out, ms_per_call);
    case 2: {
      bbrcit::GaussianProductKernel2d<float> k;
      k.set_bandwidths((float)hx, (float)hy);
      return run(k, n, xy, mass, abw, m, q, block, reps, out, ms_per_call);
    }
  }
  return 2;
}

}  // extern "C"
