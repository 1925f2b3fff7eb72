// Learned log-density surrogate: parameters, training (BF16 tensor-core forward /
// backward, FP32 Adam), inference, gradient export and persistence.
//
// No reference counterpart: the reference evaluates every query with a density
// sum. The surrogate is trained on exact densities produced by the pair-sum
// kernels and is judged against them on dense grids (bbkde_eval_grid).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/bbkde.h"
#include "mlp.cuh"
#include "mlp_tc.cuh"

using namespace bbkde::mlp;

struct bbkde_surrogate {
  int device = 0;
  cudaStream_t stream = nullptr;
  Norm norm = {0.f, 0.f, 1.f, 1.f, 0.f, 1.f};
  float *params = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr;
  __nv_bfloat16 *w2 = nullptr, *w3 = nullptr;
  float *grad_part = nullptr, *loss_part = nullptr, *loss = nullptr;
  size_t part_cap = 0;
  int64_t *index = nullptr;
  size_t index_cap = 0;
  float2 *xy = nullptr;
  float *target = nullptr;
  size_t data_cap = 0;
  float *pred = nullptr;
  size_t pred_cap = 0;
  int64_t adam_step = 0;
  int split = 0;   // inference with two-term BF16 activations
  int engine = BBKDE_ENGINE_TCGEN05;
  int *status = nullptr;   // device flag set by the tcgen05 kernel if a wait expired
  std::string err;
};

namespace bbkde {
int surrogate_check(bbkde_surrogate *s);
}  // namespace bbkde

namespace {

int sfail(bbkde_surrogate *s, int code, const std::string &m) {
  if (s) s->err = m;
  return code;
}

#define S_CUDA(s, call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return sfail(s, BBKDE_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define S_TRY(expr)                 \
  do {                              \
    int rc_ = (expr);               \
    if (rc_ != BBKDE_OK) return rc_; \
  } while (0)

template <typename T>
int grow(bbkde_surrogate *s, T *&p, size_t &cap, size_t n) {
  if (cap >= n) return BBKDE_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return sfail(s, BBKDE_ALLOC_FAILED, "cudaMalloc failed");
  }
  cap = n;
  return BBKDE_OK;
}

uint64_t splitmix(uint64_t &state) {
  uint64_t z = (state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Uniform(-a, a) initialisation with a = sqrt(6 / (fan_in + fan_out)); biases 0.
std::vector<float> init_params(uint64_t seed) {
  std::vector<float> p(kParams, 0.f);
  uint64_t st = seed;
  auto uni = [&](float a) {
    return (float)(((splitmix(st) >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0) * a;
  };
  const float a1 = std::sqrt(6.f / (2 + kH)), a2 = std::sqrt(6.f / (kH + kH)),
              a4 = std::sqrt(6.f / (kH + 1));
  for (int i = 0; i < kH * 2; ++i) p[kOffW1 + i] = uni(a1);
  for (int i = 0; i < kH * kH; ++i) p[kOffW2 + i] = uni(a2);
  for (int i = 0; i < kH * kH; ++i) p[kOffW3 + i] = uni(a2);
  for (int i = 0; i < kH; ++i) p[kOffW4 + i] = uni(a4);
  return p;
}

int refresh_bf16(bbkde_surrogate *s) {
  AdamArgs a = {};
  a.params = s->params;
  a.w2 = s->w2;
  a.w3 = s->w3;
  a.nparts = 0;
  a.step = 0;
  k_mlp_reduce<<<(kParams + 255) / 256, 256, 0, s->stream>>>(a);
  S_CUDA(s, cudaGetLastError());
  return BBKDE_OK;
}

int upload_data(bbkde_surrogate *s, int64_t n, const double *xy, const double *target) {
  S_TRY(grow(s, s->xy, s->data_cap, (size_t)n));
  std::vector<float2> hxy(n);
  for (int64_t i = 0; i < n; ++i) hxy[i] = make_float2((float)xy[2 * i], (float)xy[2 * i + 1]);
  S_CUDA(s, cudaMemcpyAsync(s->xy, hxy.data(), n * sizeof(float2), cudaMemcpyHostToDevice,
                            s->stream));
  if (target) {
    size_t cap = 0;
    if (s->target) cudaFree(s->target);
    s->target = nullptr;
    S_TRY(grow(s, s->target, cap, (size_t)n));
    std::vector<float> ht(n);
    for (int64_t i = 0; i < n; ++i) ht[i] = (float)target[i];
    S_CUDA(s, cudaMemcpyAsync(s->target, ht.data(), n * sizeof(float), cudaMemcpyHostToDevice,
                              s->stream));
  }
  S_CUDA(s, cudaStreamSynchronize(s->stream));
  return BBKDE_OK;
}

int ensure_parts(bbkde_surrogate *s, int64_t batch) {
  const size_t blocks = (size_t)((batch + kTrainPts - 1) / kTrainPts);
  if (s->part_cap < blocks) {
    if (s->grad_part) cudaFree(s->grad_part);
    if (s->loss_part) cudaFree(s->loss_part);
    s->grad_part = nullptr;
    s->loss_part = nullptr;
    s->part_cap = 0;
    if (cudaMalloc(&s->grad_part, blocks * kPartStride * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s->loss_part, blocks * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return sfail(s, BBKDE_ALLOC_FAILED, "cudaMalloc(gradient partials) failed");
    }
    s->part_cap = blocks;
  }
  return grow(s, s->index, s->index_cap, (size_t)batch);
}

TrainArgs train_args(bbkde_surrogate *s, int64_t batch) {
  TrainArgs t;
  t.params = s->params;
  t.w2 = s->w2;
  t.w3 = s->w3;
  t.norm = s->norm;
  t.xy = s->xy;
  t.target = s->target;
  t.index = s->index;
  t.batch = batch;
  t.grad_part = s->grad_part;
  t.loss_part = s->loss_part;
  return t;
}

// Gradient blocks of a batch: 128-point CTAs on tcgen05 (the default engine),
// 64-point blocks on mma.sync.
unsigned train_blocks(const bbkde_surrogate *s, int64_t batch) {
  const int pts = s->engine == BBKDE_ENGINE_TCGEN05 ? kTcTrainPts : kTrainPts;
  return (unsigned)((batch + pts - 1) / pts);
}

// One forward + backward pass over targs.batch points into the gradient
// partials (one per block); returns the number of partials.
unsigned launch_train(bbkde_surrogate *s, const TrainArgs &targs) {
  const unsigned blocks = train_blocks(s, targs.batch);
  if (s->engine == BBKDE_ENGINE_TCGEN05) {
    TcTrainArgs ta;
    ta.t = targs;
    ta.status = s->status;
    k_mlp_train_tc<<<blocks, kTcRows, TcTrainSmem::kBytes, s->stream>>>(ta);
  } else {
    k_mlp_train<<<blocks, kTrainWarps * 32, kTrainSmem, s->stream>>>(targs);
  }
  return blocks;
}

__global__ void k_iota(int64_t *idx, int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) idx[i] = i;
}

}  // namespace

extern "C" {

int bbkde_surrogate_create(int device, uint64_t seed, bbkde_surrogate **out) {
  if (!out) return BBKDE_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return BBKDE_NO_DEVICE;
  }
  if (device < 0 || device >= ndev) return BBKDE_INVALID_ARGUMENT;
  bbkde_surrogate *s = new (std::nothrow) bbkde_surrogate();
  if (!s) return BBKDE_ALLOC_FAILED;
  s->device = device;
  int rc = BBKDE_OK;
  do {
    if (cudaSetDevice(device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
      rc = BBKDE_CUDA_ERROR;
      break;
    }
    if (cudaMalloc(&s->params, kParams * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s->m, kParams * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s->v, kParams * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s->grad, kParams * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s->loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&s->w2, kH * kH * sizeof(__nv_bfloat16)) != cudaSuccess ||
        cudaMalloc(&s->w3, kH * kH * sizeof(__nv_bfloat16)) != cudaSuccess ||
        cudaMalloc(&s->status, sizeof(int)) != cudaSuccess ||
        cudaMemset(s->status, 0, sizeof(int)) != cudaSuccess) {
      rc = BBKDE_ALLOC_FAILED;
      break;
    }
    if (cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTrainSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_infer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kInferSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_infer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kInferSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_infer_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TcSmem<false>::kBytes) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_infer_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TcSmem<true>::kBytes) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TcTrainSmem::kBytes) != cudaSuccess) {
      rc = BBKDE_CUDA_ERROR;
      break;
    }
    std::vector<float> p = init_params(seed);
    if (cudaMemcpy(s->params, p.data(), kParams * sizeof(float), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemset(s->m, 0, kParams * sizeof(float)) != cudaSuccess ||
        cudaMemset(s->v, 0, kParams * sizeof(float)) != cudaSuccess) {
      rc = BBKDE_CUDA_ERROR;
      break;
    }
    if ((rc = refresh_bf16(s)) != BBKDE_OK) break;
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) rc = BBKDE_CUDA_ERROR;
  } while (0);
  if (rc != BBKDE_OK) {
    cudaGetLastError();
    bbkde_surrogate_destroy(s);
    return rc;
  }
  *out = s;
  return BBKDE_OK;
}

int bbkde_surrogate_destroy(bbkde_surrogate *s) {
  if (!s) return BBKDE_OK;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (void *p : {(void *)s->params, (void *)s->m, (void *)s->v, (void *)s->grad,
                  (void *)s->loss, (void *)s->w2, (void *)s->w3, (void *)s->grad_part,
                  (void *)s->loss_part, (void *)s->index, (void *)s->xy, (void *)s->target,
                  (void *)s->pred, (void *)s->status})
    if (p) cudaFree(p);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return BBKDE_OK;
}

const char *bbkde_surrogate_last_error(const bbkde_surrogate *s) {
  return s ? s->err.c_str() : "null surrogate";
}

int bbkde_surrogate_num_params(void) { return kParams; }

int bbkde_surrogate_set_params(bbkde_surrogate *s, const float *params, const float *norm6) {
  if (!s || !params) return BBKDE_INVALID_ARGUMENT;
  S_CUDA(s, cudaSetDevice(s->device));
  S_CUDA(s, cudaMemcpyAsync(s->params, params, kParams * sizeof(float), cudaMemcpyHostToDevice,
                            s->stream));
  if (norm6) s->norm = {norm6[0], norm6[1], norm6[2], norm6[3], norm6[4], norm6[5]};
  S_TRY(refresh_bf16(s));
  S_CUDA(s, cudaStreamSynchronize(s->stream));
  return BBKDE_OK;
}

int bbkde_surrogate_get_params(bbkde_surrogate *s, float *params, float *norm6) {
  if (!s) return BBKDE_INVALID_ARGUMENT;
  S_CUDA(s, cudaSetDevice(s->device));
  if (params)
    S_CUDA(s, cudaMemcpyAsync(params, s->params, kParams * sizeof(float),
                              cudaMemcpyDeviceToHost, s->stream));
  S_CUDA(s, cudaStreamSynchronize(s->stream));
  if (norm6) {
    norm6[0] = s->norm.cx; norm6[1] = s->norm.cy; norm6[2] = s->norm.sx;
    norm6[3] = s->norm.sy; norm6[4] = s->norm.mu; norm6[5] = s->norm.sigma;
  }
  return BBKDE_OK;
}

// Gradient of the mean squared error (normalised units) over all n points,
// one forward + backward pass, no update.
int bbkde_surrogate_gradient(bbkde_surrogate *s, int64_t n, const double *xy,
                             const double *target, float *grad, double *loss) {
  if (!s || n < 1 || !xy || !target) return BBKDE_INVALID_ARGUMENT;
  S_CUDA(s, cudaSetDevice(s->device));
  S_TRY(upload_data(s, n, xy, target));
  S_TRY(ensure_parts(s, n));
  k_iota<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(s->index, n);
  const unsigned blocks = launch_train(s, train_args(s, n));
  AdamArgs a = {};
  a.grad_part = s->grad_part;
  a.nparts = (int)blocks;
  a.loss_part = s->loss_part;
  a.params = s->params;
  a.w2 = s->w2;
  a.w3 = s->w3;
  a.grad_out = s->grad;
  a.loss_out = s->loss;
  a.step = 0;
  k_mlp_reduce<<<(kParams + 255) / 256, 256, 0, s->stream>>>(a);
  S_CUDA(s, cudaGetLastError());
  float l = 0.f;
  if (grad)
    S_CUDA(s, cudaMemcpyAsync(grad, s->grad, kParams * sizeof(float), cudaMemcpyDeviceToHost,
                              s->stream));
  S_CUDA(s, cudaMemcpyAsync(&l, s->loss, sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  S_CUDA(s, cudaStreamSynchronize(s->stream));
  S_TRY(bbkde::surrogate_check(s));
  if (loss) *loss = l;
  return BBKDE_OK;
}

// Adam on mini-batches drawn uniformly (seeded) from the n training rows.
// Inputs are normalised to [-1, 1] over their bounding box and targets to zero
// mean / unit variance (kept in the surrogate for prediction). The learning
// rate decays from lr to lr_final on a cosine schedule. Steps are captured
// into CUDA graphs of up to 100 steps each.
int bbkde_surrogate_train(bbkde_surrogate *s, int64_t n, const double *xy, const double *target,
                          const bbkde_train_config *cfg, double *final_loss) {
  if (!s || n < 2 || !xy || !target || !cfg || cfg->steps < 0 || cfg->batch < kTrainPts)
    return sfail(s, BBKDE_INVALID_ARGUMENT, "surrogate_train: bad arguments");
  S_CUDA(s, cudaSetDevice(s->device));
  double xmin = xy[0], xmax = xy[0], ymin = xy[1], ymax = xy[1], mu = 0, m2 = 0;
  for (int64_t i = 0; i < n; ++i) {
    xmin = std::min(xmin, xy[2 * i]); xmax = std::max(xmax, xy[2 * i]);
    ymin = std::min(ymin, xy[2 * i + 1]); ymax = std::max(ymax, xy[2 * i + 1]);
    mu += target[i];
  }
  mu /= n;
  for (int64_t i = 0; i < n; ++i) m2 += (target[i] - mu) * (target[i] - mu);
  const double sd = std::sqrt(m2 / n);
  s->norm.cx = (float)(0.5 * (xmin + xmax));
  s->norm.cy = (float)(0.5 * (ymin + ymax));
  s->norm.sx = (float)(2.0 / std::max(xmax - xmin, 1e-12));
  s->norm.sy = (float)(2.0 / std::max(ymax - ymin, 1e-12));
  s->norm.mu = (float)mu;
  s->norm.sigma = (float)(sd > 0 ? sd : 1.0);
  S_TRY(upload_data(s, n, xy, target));
  const int64_t batch = cfg->batch;
  S_TRY(ensure_parts(s, batch));
  const unsigned blocks = train_blocks(s, batch);
  const double b1 = cfg->beta1 > 0 ? cfg->beta1 : 0.9, b2 = cfg->beta2 > 0 ? cfg->beta2 : 0.999;
  const double eps = cfg->eps > 0 ? cfg->eps : 1e-8;
  const double lr0 = cfg->lr, lr1 = cfg->lr_final;
  const TrainArgs targs = train_args(s, batch);
  auto enqueue_step = [&](int64_t k) -> cudaError_t {
    // k: 0-based step of this call; Adam's step counter continues across calls.
    const double frac = cfg->steps > 1 ? (double)k / (double)(cfg->steps - 1) : 1.0;
    const double lr = lr1 + 0.5 * (lr0 - lr1) * (1.0 + std::cos(3.14159265358979323846 * frac));
    k_mlp_batch<<<(unsigned)((batch + 255) / 256), 256, 0, s->stream>>>(
        s->index, batch, n, cfg->seed, (uint64_t)(s->adam_step + k));
    launch_train(s, targs);
    AdamArgs a = {};
    a.grad_part = s->grad_part;
    a.nparts = (int)blocks;
    a.loss_part = s->loss_part;
    a.params = s->params;
    a.m = s->m;
    a.v = s->v;
    a.w2 = s->w2;
    a.w3 = s->w3;
    a.loss_out = s->loss;
    a.lr = (float)lr;
    a.beta1 = (float)b1;
    a.beta2 = (float)b2;
    a.eps = (float)eps;
    a.step = (int)(s->adam_step + k + 1);
    k_mlp_reduce<<<(kParams + 255) / 256, 256, 0, s->stream>>>(a);
    return cudaGetLastError();
  };
  const int64_t chunk = 100;
  for (int64_t k0 = 0; k0 < cfg->steps; k0 += chunk) {
    const int64_t k1 = std::min<int64_t>(cfg->steps, k0 + chunk);
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    S_CUDA(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int64_t k = k0; k < k1 && e == cudaSuccess; ++k) e = enqueue_step(k);
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return sfail(s, BBKDE_CUDA_ERROR, "surrogate_train: graph capture failed");
    }
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return sfail(s, BBKDE_CUDA_ERROR, cudaGetErrorString(e));
    e = cudaGraphLaunch(ge, s->stream);
    cudaGraphExecDestroy(ge);
    if (e != cudaSuccess) return sfail(s, BBKDE_CUDA_ERROR, cudaGetErrorString(e));
  }
  s->adam_step += cfg->steps;
  float l = 0.f;
  S_CUDA(s, cudaMemcpyAsync(&l, s->loss, sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  S_CUDA(s, cudaStreamSynchronize(s->stream));
  S_TRY(bbkde::surrogate_check(s));
  if (final_loss) *final_loss = l;
  return BBKDE_OK;
}

}  // extern "C"

namespace bbkde {

// Inference launch on `st`: points from xy (float2) or, with xy null, from the
// grid (gnx; gx0, gdx, gy0, gdy). Used by the dense-grid pipeline.
int surrogate_infer(bbkde_surrogate *s, cudaStream_t st, int64_t n, const float2 *xy,
                    int64_t gnx, double gx0, double gdx, double gy0, double gdy, float *out) {
  if (n == 0) return BBKDE_OK;
  InferArgs a;
  a.params = s->params;
  a.w2 = s->w2;
  a.w3 = s->w3;
  a.norm = s->norm;
  a.xy = xy;
  a.gnx = gnx > 0 ? gnx : 1;
  a.gx0 = gx0;
  a.gdx = gdx;
  a.gy0 = gy0;
  a.gdy = gdy;
  a.n = n;
  a.out = out;
  int sms = 0;
  S_CUDA(s, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
  if (sms < 1) return sfail(s, BBKDE_CUDA_ERROR, "surrogate: device reports no SMs");
  if (s->engine == BBKDE_ENGINE_TCGEN05) {
    // One CTA per SM, two 128-point tiles in flight per CTA.
    const int64_t tiles = (n + kTcRows - 1) / kTcRows;
    const int64_t want = (tiles + kTcWarpgroups - 1) / kTcWarpgroups;
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, sms));
    TcArgs ta;
    ta.in = a;
    ta.status = s->status;
    if (s->split)
      k_mlp_infer_tc<true><<<grid, kTcThreads, TcSmem<true>::kBytes, st>>>(ta);
    else
      k_mlp_infer_tc<false><<<grid, kTcThreads, TcSmem<false>::kBytes, st>>>(ta);
  } else {
    const int64_t tiles = (n + 15) / 16;
    const int64_t want = (tiles + kInferWarps - 1) / kInferWarps;
    const unsigned grid =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 8));
    if (s->split)
      k_mlp_infer<true><<<grid, kInferWarps * 32, kInferSmem, st>>>(a);
    else
      k_mlp_infer<false><<<grid, kInferWarps * 32, kInferSmem, st>>>(a);
  }
  S_CUDA(s, cudaGetLastError());
  return BBKDE_OK;
}

// After the stream has been synchronised: BBKDE_TIMEOUT if a tcgen05 kernel
// (inference or training) gave up waiting on the tensor cores (the flag is cleared).
int surrogate_check(bbkde_surrogate *s) {
  int flag = 0;
  S_CUDA(s, cudaMemcpy(&flag, s->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    cudaMemset(s->status, 0, sizeof(int));
    return sfail(s, BBKDE_TIMEOUT, "surrogate: tensor-core wait expired");
  }
  return BBKDE_OK;
}

int surrogate_device(const bbkde_surrogate *s) { return s->device; }

}  // namespace bbkde

extern "C" {

int bbkde_surrogate_set_inference(bbkde_surrogate *s, int split_activations) {
  if (!s || (split_activations != 0 && split_activations != 1)) return BBKDE_INVALID_ARGUMENT;
  s->split = split_activations;
  return BBKDE_OK;
}

int bbkde_surrogate_set_engine(bbkde_surrogate *s, int engine) {
  if (!s || (engine != BBKDE_ENGINE_TCGEN05 && engine != BBKDE_ENGINE_MMA_SYNC))
    return BBKDE_INVALID_ARGUMENT;
  s->engine = engine;
  return BBKDE_OK;
}

// Predicted log-density at device points (float2) into device floats, on the
// surrogate's stream (asynchronous).
int bbkde_surrogate_predict_device(bbkde_surrogate *s, int64_t n, const void *xy_f2,
                                   float *out) {
  if (!s || n < 0 || (n > 0 && (!xy_f2 || !out))) return BBKDE_INVALID_ARGUMENT;
  if (n == 0) return BBKDE_OK;
  S_CUDA(s, cudaSetDevice(s->device));
  return bbkde::surrogate_infer(s, s->stream, n, static_cast<const float2 *>(xy_f2), 0, 0.0,
                                0.0, 0.0, 0.0, out);
}

int bbkde_surrogate_predict(bbkde_surrogate *s, int64_t n, const double *xy, double *out) {
  if (!s || n < 0 || (n > 0 && (!xy || !out))) return BBKDE_INVALID_ARGUMENT;
  if (n == 0) return BBKDE_OK;
  S_CUDA(s, cudaSetDevice(s->device));
  float2 *dxy = nullptr;
  S_CUDA(s, cudaMalloc(&dxy, n * sizeof(float2)));
  std::vector<float2> hxy(n);
  for (int64_t i = 0; i < n; ++i) hxy[i] = make_float2((float)xy[2 * i], (float)xy[2 * i + 1]);
  int rc = BBKDE_OK;
  if (grow(s, s->pred, s->pred_cap, (size_t)n) != BBKDE_OK) rc = BBKDE_ALLOC_FAILED;
  if (rc == BBKDE_OK &&
      cudaMemcpyAsync(dxy, hxy.data(), n * sizeof(float2), cudaMemcpyHostToDevice, s->stream) !=
          cudaSuccess)
    rc = BBKDE_CUDA_ERROR;
  if (rc == BBKDE_OK) rc = bbkde_surrogate_predict_device(s, n, dxy, s->pred);
  std::vector<float> hp(n);
  if (rc == BBKDE_OK &&
      (cudaMemcpyAsync(hp.data(), s->pred, n * sizeof(float), cudaMemcpyDeviceToHost,
                       s->stream) != cudaSuccess ||
       cudaStreamSynchronize(s->stream) != cudaSuccess))
    rc = BBKDE_CUDA_ERROR;
  cudaFree(dxy);
  if (rc != BBKDE_OK) return sfail(s, rc, "surrogate_predict failed");
  S_TRY(bbkde::surrogate_check(s));
  for (int64_t i = 0; i < n; ++i) out[i] = hp[i];
  return BBKDE_OK;
}

// File: 8-byte magic "BBKDEMLP", int32 version, int32 kParams, 6 floats of
// normalisation, kParams floats (little-endian).
int bbkde_surrogate_save(bbkde_surrogate *s, const char *path) {
  if (!s || !path) return BBKDE_INVALID_ARGUMENT;
  std::vector<float> p(kParams);
  float norm6[6];
  S_TRY(bbkde_surrogate_get_params(s, p.data(), norm6));
  FILE *f = std::fopen(path, "wb");
  if (!f) return sfail(s, BBKDE_INVALID_ARGUMENT, std::string("cannot open ") + path);
  const int32_t hdr[2] = {1, kParams};
  bool ok = std::fwrite("BBKDEMLP", 1, 8, f) == 8 && std::fwrite(hdr, 4, 2, f) == 2 &&
            std::fwrite(norm6, 4, 6, f) == 6 &&
            std::fwrite(p.data(), 4, kParams, f) == (size_t)kParams;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? BBKDE_OK : sfail(s, BBKDE_INVALID_ARGUMENT, "write failed");
}

int bbkde_surrogate_load(bbkde_surrogate *s, const char *path) {
  if (!s || !path) return BBKDE_INVALID_ARGUMENT;
  FILE *f = std::fopen(path, "rb");
  if (!f) return sfail(s, BBKDE_INVALID_ARGUMENT, std::string("cannot open ") + path);
  char magic[8];
  int32_t hdr[2];
  float norm6[6];
  std::vector<float> p(kParams);
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "BBKDEMLP", 8) == 0 &&
            std::fread(hdr, 4, 2, f) == 2 && hdr[0] == 1 && hdr[1] == kParams &&
            std::fread(norm6, 4, 6, f) == 6 &&
            std::fread(p.data(), 4, kParams, f) == (size_t)kParams;
  std::fclose(f);
  if (!ok) return sfail(s, BBKDE_INVALID_ARGUMENT, "not a surrogate file of this version");
  return bbkde_surrogate_set_params(s, p.data(), norm6);
}

}  // extern "C"
