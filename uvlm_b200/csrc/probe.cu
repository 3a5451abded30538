// probe.cu -- FP32 and FP64 FMA throughput probes: the denominators of the
// N-body rooflines (the N-body kernels are bound by the FMA pipes, not by
// HBM or tensor cores, and the driver-measured peaks list only HBM and BF16
// GEMM).  The FP32 peak is the larger of a scalar FFMA probe and a packed
// FP32x2 probe (sm_100 FFMA2 issues two FMAs per lane, so its loop overhead
// fits in spare issue slots and it reaches the pipe's rate).
#include "common.cuh"

namespace uvlm {
namespace {

// 8 independent FMA chains per thread, 4096 iterations, result stored so the
// work cannot be removed.  FLOPs = 2 * 8 * 4096 per thread.
__global__ void __launch_bounds__(256) fma_probe_kernel(float* out, float seed) {
  float a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + 0.001f * (threadIdx.x + i);
  const float m = 0.999999f, c = 1e-7f;
#pragma unroll 4
  for (int it = 0; it < 4096; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fmaf(a[i], m, c);
  }
  float s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// The same with FP32x2 instructions: 8 packed chains, FLOPs = 2 * 2 * 8 * 4096.
__global__ void __launch_bounds__(256) fma2_probe_kernel(float* out, float seed) {
  float2 a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = make_float2(seed + 0.001f * (threadIdx.x + i), seed - 0.001f * i);
  const float2 m = make_float2(0.999999f, 0.999998f), c = make_float2(1e-7f, 2e-7f);
#pragma unroll 4
  for (int it = 0; it < 4096; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = __ffma2_rn(a[i], m, c);
  }
  float s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i].x + a[i].y;
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// FP64: 8 independent DFMA chains, 2048 iterations, FLOPs = 2 * 8 * 2048.
__global__ void __launch_bounds__(256) dfma_probe_kernel(float* out, double seed) {
  double a[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) a[i] = seed + 0.001 * (threadIdx.x + i);
  const double m = 0.999999999, c = 1e-12;
#pragma unroll 4
  for (int it = 0; it < 2048; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = fma(a[i], m, c);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += a[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = (float)s;
}

// Best of 5 timed launches (after one warm-up) of a probe kernel.
template <class F>
Error time_probe(int blocks, F launch, float* best_ms) {
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0);
    launch(rep);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  note_launch(6);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  (void)blocks;
  if (err != cudaSuccess) return fail(kErrCuda, cudaGetErrorString(err));
  *best_ms = best;
  return ok();
}

}  // namespace

Error measure_fp64_fma_peak(int num_sms, double* tflops) {
  const int blocks = num_sms * 8, threads = 256;
  float* out = nullptr;
  UVLM_CUDA_TRY(cudaMalloc(&out, sizeof(float) * blocks * threads));
  float ms = 0;
  const Error e = time_probe(blocks, [&](int rep) { dfma_probe_kernel<<<blocks, threads>>>(out, 1.0 + rep); }, &ms);
  cudaFree(out);
  UVLM_TRY(e);
  *tflops = 2.0 * 8 * 2048 * (double)blocks * threads / (ms * 1e-3) / 1e12;
  return ok();
}

Error measure_fp32_fma_peak(int num_sms, double* tflops) {
  const int blocks = num_sms * 8, threads = 256;
  float* out = nullptr;
  UVLM_CUDA_TRY(cudaMalloc(&out, sizeof(float) * blocks * threads));
  float ms1 = 0, ms2 = 0;
  Error e = time_probe(blocks, [&](int rep) { fma_probe_kernel<<<blocks, threads>>>(out, 1.0f + rep); }, &ms1);
  if (!e.code)
    e = time_probe(blocks, [&](int rep) { fma2_probe_kernel<<<blocks, threads>>>(out, 1.0f + rep); }, &ms2);
  cudaFree(out);
  UVLM_TRY(e);
  const double t1 = 2.0 * 8 * 4096 * (double)blocks * threads / (ms1 * 1e-3) / 1e12;
  const double t2 = 2.0 * 2 * 8 * 4096 * (double)blocks * threads / (ms2 * 1e-3) / 1e12;
  *tflops = t1 > t2 ? t1 : t2;
  return ok();
}

}  // namespace uvlm
