// mlp_api.cu -- C-ABI of the warm-start MLP: creation, parameters,
// normalisation, forward, gradients (for checks against autograd) and
// training on (features, target) pairs collected from the solver.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <numeric>
#include <random>
#include <vector>

#include "../../include/uvlm_b200.h"
#include "mlp.cuh"

using namespace uvlm;

struct uvlm_mlp {
  Mlp m;
};

namespace uvlm {
Mlp* mlp_of(uvlm_mlp* h) { return h ? &h->m : nullptr; }
}  // namespace uvlm

namespace {

int report(const Error& e) {
  if (e.code) set_global_error(e.msg);
  return e.code;
}

__global__ void gather_rows(const float* src, int width, const long long* idx, long long n, float* dst) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n * width; q += (long long)gridDim.x * blockDim.x) {
    const long long r = q / width;
    dst[q] = src[idx[r] * width + q % width];
  }
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
};

}  // namespace

extern "C" {

int uvlm_mlp_create(uint64_t seed, uvlm_mlp** out) {
  if (!out) return report(fail(kErrInvalid, "NULL argument"));
  auto* h = new uvlm_mlp();
  Error e = mlp_create(&h->m, seed);
  if (e.code) {
    delete h;
    return report(e);
  }
  *out = h;
  return UVLM_OK;
}

int uvlm_mlp_destroy(uvlm_mlp* h) {
  if (h) {
    mlp_free(&h->m);
    delete h;
  }
  return UVLM_OK;
}

int64_t uvlm_mlp_num_params(const uvlm_mlp* h) { return h ? (int64_t)h->m.n_params : 0; }

int uvlm_mlp_get_params(const uvlm_mlp* h, float* params) {
  if (!h || !params) return report(fail(kErrInvalid, "NULL argument"));
  if (cudaMemcpy(params, h->m.master, sizeof(float) * h->m.n_params, cudaMemcpyDeviceToHost) != cudaSuccess)
    return report(fail(kErrCuda, "parameter copy failed"));
  return UVLM_OK;
}

int uvlm_mlp_set_params(uvlm_mlp* h, const float* params) {
  if (!h || !params) return report(fail(kErrInvalid, "NULL argument"));
  if (cudaMemcpy(h->m.master, params, sizeof(float) * h->m.n_params, cudaMemcpyHostToDevice) != cudaSuccess)
    return report(fail(kErrCuda, "parameter copy failed"));
  return report(mlp_sync_bf16(&h->m, 0));
}

int uvlm_mlp_set_normalization(uvlm_mlp* h, const float* mean, const float* stdev, float out_scale) {
  if (!h || !mean || !stdev || !(out_scale > 0)) return report(fail(kErrInvalid, "invalid argument"));
  for (int f = 0; f < kMlpIn; ++f) {
    if (!(stdev[f] > 0)) return report(fail(kErrInvalid, "standard deviations must be positive"));
    h->m.h_norm[f] = mean[f];
    h->m.h_norm[kMlpIn + f] = stdev[f];
  }
  h->m.h_norm[2 * kMlpIn] = out_scale;
  if (cudaMemcpy(h->m.norm, h->m.h_norm, sizeof(h->m.h_norm), cudaMemcpyHostToDevice) != cudaSuccess)
    return report(fail(kErrCuda, "normalisation copy failed"));
  return UVLM_OK;
}

int uvlm_mlp_forward(uvlm_mlp* h, const float* x, int64_t n, float* y) {
  if (!h || !x || !y || n < 0) return report(fail(kErrInvalid, "invalid argument"));
  if (n == 0) return UVLM_OK;
  auto run = [&]() -> Error {
    DevBuf dx, dy;
    UVLM_CUDA_TRY(cudaMalloc(&dx.p, sizeof(float) * n * kMlpIn));
    UVLM_CUDA_TRY(cudaMalloc(&dy.p, sizeof(float) * n));
    UVLM_CUDA_TRY(cudaMemcpy(dx.p, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice));
    UVLM_TRY(mlp_forward(&h->m, (const float*)dx.p, n, (float*)dy.p, 0));
    UVLM_CUDA_TRY(cudaMemcpy(y, dy.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_mlp_forward_tc(uvlm_mlp* h, const float* x, int64_t n, float* y) {
  if (!h || !x || !y || n < 0 || n > INT32_MAX) return report(fail(kErrInvalid, "invalid argument"));
  if (n == 0) return UVLM_OK;
  if (!mlp_tc_available()) return report(fail(kErrUnsupported, "tcgen05 inference needs an sm_100 device"));
  auto run = [&]() -> Error {
    DevBuf dx, dy;
    UVLM_CUDA_TRY(cudaMalloc(&dx.p, sizeof(float) * n * kMlpIn));
    UVLM_CUDA_TRY(cudaMalloc(&dy.p, sizeof(float) * n));
    UVLM_CUDA_TRY(cudaMemcpy(dx.p, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice));
    UVLM_TRY(mlp_forward_tc(&h->m, (const float*)dx.p, n, (float*)dy.p, 0));
    UVLM_TRY(mlp_tc_check(&h->m, 0));
    UVLM_CUDA_TRY(cudaMemcpy(y, dy.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_mlp_gradients(uvlm_mlp* h, const float* x, const float* target, int64_t n, float* grads, double* loss) {
  if (!h || !x || !target || !grads || n < 1) return report(fail(kErrInvalid, "invalid argument"));
  auto run = [&]() -> Error {
    DevBuf dx, dt;
    UVLM_CUDA_TRY(cudaMalloc(&dx.p, sizeof(float) * n * kMlpIn));
    UVLM_CUDA_TRY(cudaMalloc(&dt.p, sizeof(float) * n));
    UVLM_CUDA_TRY(cudaMemcpy(dx.p, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice));
    UVLM_CUDA_TRY(cudaMemcpy(dt.p, target, sizeof(float) * n, cudaMemcpyHostToDevice));
    double l = 0;
    UVLM_TRY(mlp_loss_backward(&h->m, (const float*)dx.p, (const float*)dt.p, n, &l, 0));
    UVLM_CUDA_TRY(cudaMemcpy(grads, h->m.grad, sizeof(float) * h->m.n_params, cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    return ok();
  };
  return report(run());
}

int uvlm_mlp_train(uvlm_mlp* h, const float* x, const float* target, int64_t n, int32_t epochs, int32_t batch,
                   double lr, uint64_t seed, double* final_loss) {
  if (!h || !x || !target || n < 1 || epochs < 1 || batch < 1 || !(lr > 0))
    return report(fail(kErrInvalid, "invalid argument"));
  auto run = [&]() -> Error {
    DevBuf dx, dt, bx, bt, didx;
    UVLM_CUDA_TRY(cudaMalloc(&dx.p, sizeof(float) * n * kMlpIn));
    UVLM_CUDA_TRY(cudaMalloc(&dt.p, sizeof(float) * n));
    UVLM_CUDA_TRY(cudaMalloc(&bx.p, sizeof(float) * (size_t)batch * kMlpIn));
    UVLM_CUDA_TRY(cudaMalloc(&bt.p, sizeof(float) * (size_t)batch));
    UVLM_CUDA_TRY(cudaMalloc(&didx.p, sizeof(long long) * n));
    UVLM_CUDA_TRY(cudaMemcpy(dx.p, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice));
    UVLM_CUDA_TRY(cudaMemcpy(dt.p, target, sizeof(float) * n, cudaMemcpyHostToDevice));
    std::vector<long long> idx(n);
    std::iota(idx.begin(), idx.end(), 0LL);
    std::mt19937_64 rng(seed);
    double epoch_loss = 0;
    for (int e = 0; e < epochs; ++e) {
      std::shuffle(idx.begin(), idx.end(), rng);
      UVLM_CUDA_TRY(cudaMemcpy(didx.p, idx.data(), sizeof(long long) * n, cudaMemcpyHostToDevice));
      epoch_loss = 0;
      long long nb = 0;
      for (long long b0 = 0; b0 + batch <= n || (b0 == 0 && n < batch); b0 += batch) {
        const long long B = std::min<long long>(batch, n - b0);
        const long long* ib = (const long long*)didx.p + b0;
        gather_rows<<<std::min<long long>((B * kMlpIn + 255) / 256, 4096), 256>>>((const float*)dx.p, kMlpIn, ib, B,
                                                                                (float*)bx.p);
        UVLM_LAUNCH_CHECK();
        gather_rows<<<std::min<long long>((B + 255) / 256, 4096), 256>>>((const float*)dt.p, 1, ib, B, (float*)bt.p);
        UVLM_LAUNCH_CHECK();
        double l = 0;
        UVLM_TRY(mlp_loss_backward(&h->m, (const float*)bx.p, (const float*)bt.p, B, &l, 0));
        UVLM_TRY(mlp_adam_step(&h->m, (float)lr, 0));
        epoch_loss += l;
        ++nb;
      }
      if (nb) epoch_loss /= (double)nb;
    }
    UVLM_CUDA_TRY(cudaDeviceSynchronize());
    if (final_loss) *final_loss = epoch_loss;
    return ok();
  };
  return report(run());
}

}  // extern "C"
