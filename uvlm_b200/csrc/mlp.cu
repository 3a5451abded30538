// mlp.cu -- hand-written forward / backward / Adam kernels of the warm-start MLP.
#include <cmath>
#include <random>
#include <vector>

#include "mlp.cuh"

namespace uvlm {
namespace {

constexpr float kInvSqrt2 = 0.70710678118654752f;
constexpr float kInvSqrt2Pi = 0.39894228040143268f;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * kInvSqrt2)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * kInvSqrt2)) + z * kInvSqrt2Pi * __expf(-0.5f * z * z);
}

// Tiled FP32-accumulate product, 64 x 64 output tile per 256-thread CTA,
// 4 x 4 outputs per thread, inner dimension staged 32 at a time:
//   C[r][c] = sum_i A'(i, r) * B'(i, c)
// MODE 0 (forward):      A' = X[r][i] (ld K),  B' = W[i][c] (bf16, ld N)
// MODE 1 (backward-data): A' = dZ[r][i] (ld N), B' = W[c][i] (bf16, ld N)
// MODE 2 (weight grad):  A' = Aprev[i][r] (ld K), B' = dZ[i][c] (ld N)
// EPI 0: C = acc; EPI 1: Z = acc + bias, A = GELU(Z); EPI 2: C = acc * GELU'(Zp[r][c])
template <int MODE, int EPI>
__global__ void __launch_bounds__(256) mlp_gemm(const float* __restrict__ A, const __nv_bfloat16* __restrict__ Wb,
                                                const float* __restrict__ Bf, int rows, int cols, int inner, int lda,
                                                int ldb, const float* __restrict__ bias, const float* __restrict__ Zp,
                                                float* __restrict__ C, float* __restrict__ Cact, int ldc) {
  __shared__ float As[32][64];
  __shared__ float Bs[32][64];
  const int row0 = blockIdx.y * 64, col0 = blockIdx.x * 64;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  float acc[4][4] = {};
  for (int i0 = 0; i0 < inner; i0 += 32) {
    for (int q = tid; q < 32 * 64; q += 256) {
      const int ii = q / 64, r = q % 64;
      const int i = i0 + ii, R = row0 + r;
      float v = 0.f;
      if (i < inner && R < rows) {
        if (MODE == 2)
          v = A[(long long)i * lda + R];
        else
          v = A[(long long)R * lda + i];
      }
      As[ii][r] = v;
      const int Cc = col0 + r;
      float w = 0.f;
      if (i < inner && Cc < cols) {
        if (MODE == 0) w = __bfloat162float(Wb[(long long)i * ldb + Cc]);
        if (MODE == 1) w = __bfloat162float(Wb[(long long)Cc * ldb + i]);
        if (MODE == 2) w = Bf[(long long)i * ldb + Cc];
      }
      Bs[ii][r] = w;
    }
    __syncthreads();
#pragma unroll 8
    for (int ii = 0; ii < 32; ++ii) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = As[ii][ty * 4 + u];
#pragma unroll
      for (int u = 0; u < 4; ++u) b[u] = Bs[ii][tx * 4 + u];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int R = row0 + ty * 4 + u;
    if (R >= rows) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int Cc = col0 + tx * 4 + v;
      if (Cc >= cols) continue;
      const long long o = (long long)R * ldc + Cc;
      if (EPI == 0) C[o] = acc[u][v];
      if (EPI == 1) {
        const float z = acc[u][v] + bias[Cc];
        C[o] = z;
        Cact[o] = gelu(z);
      }
      if (EPI == 2) C[o] = acc[u][v] * gelu_grad(Zp[o]);
    }
  }
}

// last layer (out = 1): y[b] = out_scale * (A[b] . w + b0), warp per row
__global__ void head_forward(const float* __restrict__ A, int B, int K, const __nv_bfloat16* __restrict__ w,
                             const float* __restrict__ b0, const float* __restrict__ norm, float* y) {
  const int lane = threadIdx.x & 31;
  const long long row = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (row >= B) return;
  float s = 0;
  for (int k = lane; k < K; k += 32) s += A[row * K + k] * __bfloat162float(w[k]);
  for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (lane == 0) y[row] = (s + b0[0]) * norm[2 * kMlpIn];
}

// x' = (x - mean) / std into act[0] (ld kMlpIn)
__global__ void normalise_inputs(const float* __restrict__ x, long long B, const float* __restrict__ norm, float* a0) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < B * kMlpIn; q += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(q % kMlpIn);
    a0[q] = (x[q] - norm[f]) / norm[kMlpIn + f];
  }
}

// dy = 2 (y - t) / (B s^2) on the network output scale; loss partial sums
__global__ void loss_grad(const float* __restrict__ y, const float* __restrict__ t, long long B,
                          const float* __restrict__ norm, float* dy, double* loss) {
  __shared__ double sh[8];
  const float s = norm[2 * kMlpIn];
  double acc = 0;
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < B; b += (long long)gridDim.x * blockDim.x) {
    const float e = (y[b] - t[b]) / s;  // error in network units
    acc += (double)e * e;
    dy[b] = 2.f * e / (float)B;
  }
  for (int off = 16; off; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    for (int i = 0; i < (int)(blockDim.x / 32); ++i) v += sh[i];
    atomicAdd(loss, v / (double)B);
  }
}

// head backward: dW4[k] = sum_b A[b][k] dy[b]; db4 = sum_b dy[b];
// dZ3[b][k] = dy[b] * w[k] * GELU'(Z3[b][k])
__global__ void head_backward_data(const float* __restrict__ dy, long long B, int K, const __nv_bfloat16* __restrict__ w,
                                   const float* __restrict__ Z, float* dZ) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < B * K; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % K);
    const long long b = q / K;
    dZ[q] = dy[b] * __bfloat162float(w[k]) * gelu_grad(Z[q]);
  }
}

// column sums: out[c] = sum_b M[b][c] * (wvec ? wvec[b] : 1)
__global__ void column_sums(const float* __restrict__ M, long long B, int cols, const float* __restrict__ wvec,
                            float* out) {
  const int c = blockIdx.x;
  double s = 0;
  for (long long b = threadIdx.x; b < B; b += blockDim.x) s += (double)M[b * cols + c] * (wvec ? wvec[b] : 1.f);
  __shared__ double sh[8];
  for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0;
    for (int i = 0; i < (int)(blockDim.x / 32); ++i) v += sh[i];
    out[c] = (float)v;
  }
}

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2, __nv_bfloat16* pb) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float upd = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    const float pi = p[i] - upd;
    p[i] = pi;
    pb[i] = __float2bfloat16(pi);
  }
}

__global__ void to_bf16(const float* p, size_t n, __nv_bfloat16* pb) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    pb[i] = __float2bfloat16(p[i]);
}

__global__ void features_kernel(int num, int R, int C, const double* g_n, const double* g_nm1, const double* b_np1,
                                const double* b_n, const double* phase, float* feat) {
  const int per = R * C;
  const int N = per * num;
  for (int K = blockIdx.x * blockDim.x + threadIdx.x; K < N; K += gridDim.x * blockDim.x) {
    const int n = K / per, i = (K % per) / C, j = K % C;
    float* f = feat + (long long)K * kMlpIn;
    f[0] = (float)g_n[K];
    f[1] = (float)(g_n[K] - g_nm1[K]);
    f[2] = (float)b_np1[K];
    f[3] = (float)(b_np1[K] - b_n[K]);
    f[4] = (float)sin(phase[n]);
    f[5] = (float)cos(phase[n]);
    f[6] = 2.f * (i + 0.5f) / R - 1.f;
    f[7] = 2.f * (j + 0.5f) / C - 1.f;
  }
}

__global__ void guess_kernel(int N, const double* g_n, const double* g_nm1, const float* y, double* x0) {
  for (int K = blockIdx.x * blockDim.x + threadIdx.x; K < N; K += gridDim.x * blockDim.x)
    x0[K] = 2.0 * g_n[K] - g_nm1[K] + (double)y[K];
}

__global__ void targets_kernel(int N, const double* g_np1, const double* g_n, const double* g_nm1, float* t) {
  for (int K = blockIdx.x * blockDim.x + threadIdx.x; K < N; K += gridDim.x * blockDim.x)
    t[K] = (float)(g_np1[K] - (2.0 * g_n[K] - g_nm1[K]));
}

inline int g1(long long n) { return (int)std::min<long long>(std::max<long long>((n + 255) / 256, 1), 8192); }

}  // namespace

Error mlp_create(Mlp* m, unsigned long long seed) {
  mlp_free(m);
  const int dims[kMlpDepth + 2] = {kMlpIn, kMlpHidden, kMlpHidden, kMlpHidden, 1};
  size_t off = 0;
  for (int l = 0; l <= kMlpDepth; ++l) {
    m->layer[l].in = dims[l];
    m->layer[l].out = dims[l + 1];
    m->layer[l].w_off = off;
    off += (size_t)dims[l] * dims[l + 1];
    m->layer[l].b_off = off;
    off += dims[l + 1];
  }
  m->n_params = off;
  std::vector<float> p(off, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l <= kMlpDepth; ++l) {
    const float lim = std::sqrt(3.0f / (float)m->layer[l].in) * (l == kMlpDepth ? 0.1f : 1.0f);
    std::uniform_real_distribution<float> U(-lim, lim);
    for (size_t q = 0; q < (size_t)m->layer[l].in * m->layer[l].out; ++q) p[m->layer[l].w_off + q] = U(rng);
  }
  UVLM_CUDA_TRY(cudaMalloc(&m->master, sizeof(float) * off));
  UVLM_CUDA_TRY(cudaMalloc(&m->wbf, sizeof(__nv_bfloat16) * off));
  UVLM_CUDA_TRY(cudaMalloc(&m->grad, sizeof(float) * off));
  UVLM_CUDA_TRY(cudaMalloc(&m->adam_m, sizeof(float) * off));
  UVLM_CUDA_TRY(cudaMalloc(&m->adam_v, sizeof(float) * off));
  UVLM_CUDA_TRY(cudaMalloc(&m->norm, sizeof(float) * (2 * kMlpIn + 1)));
  UVLM_CUDA_TRY(cudaMalloc(&m->loss, sizeof(double)));
  UVLM_CUDA_TRY(cudaMemcpy(m->master, p.data(), sizeof(float) * off, cudaMemcpyHostToDevice));
  UVLM_CUDA_TRY(cudaMemset(m->adam_m, 0, sizeof(float) * off));
  UVLM_CUDA_TRY(cudaMemset(m->adam_v, 0, sizeof(float) * off));
  for (int f = 0; f < kMlpIn; ++f) {
    m->h_norm[f] = 0.f;
    m->h_norm[kMlpIn + f] = 1.f;
  }
  m->h_norm[2 * kMlpIn] = 1.f;
  UVLM_CUDA_TRY(cudaMemcpy(m->norm, m->h_norm, sizeof(m->h_norm), cudaMemcpyHostToDevice));
  m->adam_t = 0;
  return mlp_sync_bf16(m, 0);
}

void mlp_free(Mlp* m) {
  cudaFree(m->master);
  cudaFree(m->wbf);
  cudaFree(m->grad);
  cudaFree(m->adam_m);
  cudaFree(m->adam_v);
  cudaFree(m->norm);
  cudaFree(m->loss);
  cudaFree(m->act);
  cudaFree(m->pre);
  cudaFree(m->dact);
  cudaFree(m->y);
  cudaFree(m->dy);
  cudaFree(m->wT);
  cudaFree(m->tc_err);
  *m = Mlp{};
}

Error mlp_reserve(Mlp* m, long long B) {
  if (B <= m->cap) return ok();
  cudaFree(m->act);
  cudaFree(m->pre);
  cudaFree(m->dact);
  cudaFree(m->y);
  cudaFree(m->dy);
  m->act = m->pre = m->dact = m->y = m->dy = nullptr;
  const size_t H = kMlpHidden;
  UVLM_CUDA_TRY(cudaMalloc(&m->act, sizeof(float) * (kMlpDepth + 1) * B * H));
  UVLM_CUDA_TRY(cudaMalloc(&m->pre, sizeof(float) * kMlpDepth * B * H));
  UVLM_CUDA_TRY(cudaMalloc(&m->dact, sizeof(float) * 2 * B * H));
  UVLM_CUDA_TRY(cudaMalloc(&m->y, sizeof(float) * B));
  UVLM_CUDA_TRY(cudaMalloc(&m->dy, sizeof(float) * B));
  m->cap = B;
  return ok();
}

Error mlp_sync_bf16(Mlp* m, cudaStream_t st) {
  m->version += 1;
  to_bf16<<<g1((long long)m->n_params), 256, 0, st>>>(m->master, m->n_params, m->wbf);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error mlp_forward(Mlp* m, const float* x, long long B, float* y, cudaStream_t st) {
  if (B <= 0) return ok();
  UVLM_TRY(mlp_reserve(m, B));
  const long long H = kMlpHidden;
  normalise_inputs<<<g1(B * kMlpIn), 256, 0, st>>>(x, B, m->norm, m->act);
  UVLM_LAUNCH_CHECK();
  for (int l = 0; l < kMlpDepth; ++l) {
    const MlpLayer& L = m->layer[l];
    const float* Ain = m->act + (long long)l * B * H;
    float* Z = m->pre + (long long)l * B * H;
    float* Aout = m->act + (long long)(l + 1) * B * H;
    dim3 grid(ceil_div(L.out, 64), ceil_div(B, 64));
    mlp_gemm<0, 1><<<grid, 256, 0, st>>>(Ain, m->wbf + L.w_off, nullptr, (int)B, L.out, L.in, L.in, L.out,
                                         m->master + L.b_off, nullptr, Z, Aout, L.out);
    UVLM_LAUNCH_CHECK();
  }
  const MlpLayer& Lh = m->layer[kMlpDepth];
  head_forward<<<ceil_div(B, 8), 256, 0, st>>>(m->act + (long long)kMlpDepth * B * H, (int)B, Lh.in,
                                               m->wbf + Lh.w_off, m->master + Lh.b_off, m->norm, y ? y : m->y);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error mlp_loss_backward(Mlp* m, const float* x, const float* target, long long B, double* loss_host,
                        cudaStream_t st) {
  UVLM_TRY(mlp_forward(m, x, B, m->y, st));
  const long long H = kMlpHidden;
  UVLM_CUDA_TRY(cudaMemsetAsync(m->loss, 0, sizeof(double), st));
  loss_grad<<<std::min(g1(B), 1024), 256, 0, st>>>(m->y, target, B, m->norm, m->dy, m->loss);
  UVLM_LAUNCH_CHECK();
  // head: dW4 = A3^T dy, db4 = sum dy, dZ3 = dy w4 GELU'(Z3)
  const MlpLayer& Lh = m->layer[kMlpDepth];
  const float* A3 = m->act + (long long)kMlpDepth * B * H;
  column_sums<<<Lh.in, 256, 0, st>>>(A3, B, Lh.in, m->dy, m->grad + Lh.w_off);
  UVLM_LAUNCH_CHECK();
  column_sums<<<1, 256, 0, st>>>(m->dy, B, 1, nullptr, m->grad + Lh.b_off);
  UVLM_LAUNCH_CHECK();
  float* dZ = m->dact;            // dZ of the current layer
  float* dZnext = m->dact + B * H;
  head_backward_data<<<g1(B * Lh.in), 256, 0, st>>>(m->dy, B, Lh.in, m->wbf + Lh.w_off,
                                                    m->pre + (long long)(kMlpDepth - 1) * B * H, dZ);
  UVLM_LAUNCH_CHECK();
  for (int l = kMlpDepth - 1; l >= 0; --l) {
    const MlpLayer& L = m->layer[l];
    const float* Ain = m->act + (long long)l * B * H;
    // dW = Ain^T dZ  [in x out], db = column sums of dZ
    dim3 gw(ceil_div(L.out, 64), ceil_div(L.in, 64));
    mlp_gemm<2, 0><<<gw, 256, 0, st>>>(Ain, nullptr, dZ, L.in, L.out, (int)B, L.in, L.out, nullptr, nullptr,
                                       m->grad + L.w_off, nullptr, L.out);
    UVLM_LAUNCH_CHECK();
    column_sums<<<L.out, 256, 0, st>>>(dZ, B, L.out, nullptr, m->grad + L.b_off);
    UVLM_LAUNCH_CHECK();
    if (l > 0) {
      // dZ_{l-1} = (dZ W^T) * GELU'(Z_{l-1})
      dim3 gd(ceil_div(L.in, 64), ceil_div(B, 64));
      mlp_gemm<1, 2><<<gd, 256, 0, st>>>(dZ, m->wbf + L.w_off, nullptr, (int)B, L.in, L.out, L.out, L.out, nullptr,
                                         m->pre + (long long)(l - 1) * B * H, dZnext, nullptr, L.in);
      UVLM_LAUNCH_CHECK();
      std::swap(dZ, dZnext);
    }
  }
  if (loss_host) {
    UVLM_CUDA_TRY(cudaMemcpyAsync(loss_host, m->loss, sizeof(double), cudaMemcpyDeviceToHost, st));
    UVLM_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return ok();
}

Error mlp_adam_step(Mlp* m, float lr, cudaStream_t st) {
  m->adam_t += 1;
  m->version += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - (float)std::pow(b1, (double)m->adam_t);
  const float c2 = 1.f - (float)std::pow(b2, (double)m->adam_t);
  adam_kernel<<<g1((long long)m->n_params), 256, 0, st>>>(m->master, m->grad, m->adam_m, m->adam_v, m->n_params, lr,
                                                          b1, b2, 1e-8f, c1, c2, m->wbf);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error mlp_features(int num, int R, int C, const double* g_n, const double* g_nm1, const double* b_np1,
                   const double* b_n, const double* phase, float* feat, cudaStream_t st) {
  features_kernel<<<g1((long long)num * R * C), 256, 0, st>>>(num, R, C, g_n, g_nm1, b_np1, b_n, phase, feat);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error mlp_apply_guess(int N, const double* g_n, const double* g_nm1, const float* y, double* x0, cudaStream_t st) {
  guess_kernel<<<g1(N), 256, 0, st>>>(N, g_n, g_nm1, y, x0);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error mlp_targets(int N, const double* g_np1, const double* g_n, const double* g_nm1, float* t, cudaStream_t st) {
  targets_kernel<<<g1(N), 256, 0, st>>>(N, g_np1, g_n, g_nm1, t);
  UVLM_LAUNCH_CHECK();
  return ok();
}

}  // namespace uvlm
