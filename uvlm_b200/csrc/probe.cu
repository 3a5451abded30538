// probe.cu -- FP32 FMA throughput probe: the denominator of the N-body
// roofline (the N-body kernels are bound by FP32 SIMT issue, not by HBM or
// tensor cores, and the driver-measured peaks list only HBM and BF16 GEMM).
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

}  // namespace

Error measure_fp32_fma_peak(int num_sms, double* tflops) {
  const int blocks = num_sms * 8, threads = 256;
  float* out = nullptr;
  UVLM_CUDA_TRY(cudaMalloc(&out, sizeof(float) * blocks * threads));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0);
    fma_probe_kernel<<<blocks, threads>>>(out, 1.0f + rep);
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
  cudaFree(out);
  if (err != cudaSuccess) return fail(kErrCuda, cudaGetErrorString(err));
  const double flops = 2.0 * 8 * 4096 * (double)blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return ok();
}

}  // namespace uvlm
