// mlp.cuh -- the learned warm start of the circulation solve.
//
// No counterpart in the reference.  A per-panel MLP maps
//   (G_n, G_n - G_{n-1}, b_{n+1}, b_{n+1} - b_n, sin phi, cos phi, x, y)
// (x, y: the panel's chordwise/spanwise position in [-1, 1]) to a correction
// of the linear extrapolation 2 G_n - G_{n-1} of the panel's circulation, and
// the result is the initial guess of the stale-LU-preconditioned GMRES solve.
// Hidden layers: kMlpDepth x kMlpHidden with GELU; weights are used in BF16
// (FP32 masters for Adam), all products accumulate in FP32.  Forward, backward
// and Adam are hand-written kernels.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

#include "common.cuh"

namespace uvlm {

constexpr int kMlpIn = 8;
constexpr int kMlpHidden = 256;
constexpr int kMlpDepth = 3;  // hidden layers

struct MlpLayer {
  int in, out;
  size_t w_off, b_off;  // offsets (floats) into the parameter vector: W [in][out], b [out]
};

struct Mlp {
  int n_layers = kMlpDepth + 1;
  MlpLayer layer[kMlpDepth + 1];
  size_t n_params = 0;
  float* master = nullptr;     // FP32 parameters
  __nv_bfloat16* wbf = nullptr;  // BF16 copy used by the products (same offsets)
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  long long adam_t = 0;
  // normalisation: x' = (x - mean) / std per feature, y = out_scale * net(x')
  float* norm = nullptr;  // [2 * kMlpIn + 1] on the device
  float h_norm[2 * kMlpIn + 1];
  // activations cache for training / inference
  long long cap = 0;
  float* act = nullptr;   // [depth+1][cap][hidden]: layer inputs
  float* pre = nullptr;   // [depth][cap][hidden]: pre-activations
  float* dact = nullptr;  // [2][cap][hidden]
  float* y = nullptr;     // [cap]
  float* dy = nullptr;    // [cap]
  double* loss = nullptr; // [1]
  // tensor-core inference (mlp_tc.cu): K-major BF16 copies of the two hidden
  // 256 x 256 weight matrices and their TMA maps, rebuilt when the weights
  // change (version counts the changes of wbf)
  long long version = 0, wT_version = -1;
  __nv_bfloat16* wT = nullptr;  // [2][256][256]
  CUtensorMap tmap[2];
  int* tc_err = nullptr;        // a bounded wait of the inference kernel gave up
};

Error mlp_create(Mlp* m, unsigned long long seed);
void mlp_free(Mlp* m);
Error mlp_reserve(Mlp* m, long long batch);
// y[b] = out_scale * net((x[b] - mean) / std), x: [B][kMlpIn] FP32 device
Error mlp_forward(Mlp* m, const float* x, long long B, float* y, cudaStream_t st);
// loss = mean (y - target)^2 and gradients of all parameters into m->grad
Error mlp_loss_backward(Mlp* m, const float* x, const float* target, long long B, double* loss_host,
                        cudaStream_t st);
Error mlp_adam_step(Mlp* m, float lr, cudaStream_t st);
Error mlp_sync_bf16(Mlp* m, cudaStream_t st);

// Tensor-core inference (tcgen05, BF16 operands, FP32 accumulation), fused:
// y = out_scale * net((x - mean)/std) for feature rows x [B][kMlpIn] ...
Error mlp_forward_tc(Mlp* m, const float* x, long long B, float* y, cudaStream_t st);
// ... or straight from the solver state (the features of mlp_features) to
// the initial guess x0 = 2 g_n - g_{n-1} + y of every panel.
Error mlp_guess_tc(Mlp* m, int num, int R, int C, const double* g_n, const double* g_nm1, const double* b_np1,
                   const double* b_n, const double* phase, double* x0, cudaStream_t st);
// UVLM_ERR_TIMEOUT if a bounded wait of the inference kernel gave up since
// the last check (synchronises the stream).
Error mlp_tc_check(Mlp* m, cudaStream_t st);
bool mlp_tc_available();
Error mlp_tc_set_wait_limit(long long cycles);

// Features of all N panels for predicting step n+1 (see the header comment),
// written as [N][kMlpIn] FP32.  phase[n] = phase of wing n at t_{n+1}.
Error mlp_features(int num, int R, int C, const double* g_n, const double* g_nm1, const double* b_np1,
                   const double* b_n, const double* phase, float* feat, cudaStream_t st);
// x0 = 2 g_n - g_{n-1} + y
Error mlp_apply_guess(int N, const double* g_n, const double* g_nm1, const float* y, double* x0, cudaStream_t st);
// training target: (g_{n+1} - (2 g_n - g_{n-1}))
Error mlp_targets(int N, const double* g_np1, const double* g_n, const double* g_nm1, float* t, cudaStream_t st);

}  // namespace uvlm
