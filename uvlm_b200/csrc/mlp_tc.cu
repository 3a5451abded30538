// mlp_tc.cu -- inference of the warm-start MLP on the tcgen05 tensor cores,
// fused with its features and the initial guess of the solve.
//
// One CTA (128 threads) evaluates 128 panels, thread t owning panel row t:
//   1. features of its panel (or a given feature row), normalised; layer 1
//      (8 -> 256, FP32 on the CUDA cores: K = 8 is below one MMA step) with
//      GELU, rounded to BF16 into a K-major, 128-byte-swizzled activation
//      tile [128 x 256] in shared memory;
//   2. layer 2: one elected thread issues 16 tcgen05.mma (kind::f16, BF16
//      operands, M = 128, N = 256, K = 16 each) against W2^T, brought in by
//      TMA while layer 1 ran; the FP32 accumulator lives in TMEM (256 columns);
//   3. the four warps read their 32 accumulator rows back (tcgen05.ld), add
//      the bias, apply GELU and write BF16 activations over the layer-1 tile
//      while TMA brings W3^T over W2^T;
//   4. layer 3 the same way;
//   5. the head (256 -> 1) straight from TMEM: bias, GELU, dot with the
//      output weights in FP32; y = out_scale * (dot + b4), and the guess
//      x0 = 2 g_n - g_{n-1} + y in FP64.
// The activations of layers 2-3 are BF16 (the MMA takes BF16 operands) and
// GELU takes its tanh form, so the prediction differs from the SIMT forward
// (FP32 activations, erf form) at the BF16 level; it only seeds the GMRES
// solve, whose answer is the same.
// Every wait is bounded (g_wait_limit); on a timeout the CTA raises err[0],
// waits (bounded) for its own TMA copies and MMAs in flight, frees its TMEM
// and returns.
#include <cuda.h>
#include <cuda_bf16.h>

#include "lu.cuh"
#include "mlp.cuh"
#include "tc_common.cuh"

namespace uvlm {
namespace {

constexpr int kRows = 128;                          // panels per CTA: the MMA's M
constexpr int kH = kMlpHidden;                      // 256: N and K of the hidden layers
constexpr int kKChunks = kH / 64;                   // 128-byte swizzle rows of K (64 BF16 each)
constexpr size_t kActChunk = (size_t)kRows * 128;   // 16 KB
constexpr size_t kWChunk = (size_t)kH * 128;        // 32 KB
constexpr size_t kActBytes = kKChunks * kActChunk;  // 64 KB
constexpr size_t kWBytes = kKChunks * kWChunk;      // 128 KB
// small operands staged as FP32: W1 [8][256], b1, b2, b3, w4
constexpr size_t kSmallFloats = (size_t)kMlpIn * kH + 4 * kH;
constexpr size_t kSmemBytes = 1024 + kActBytes + kWBytes + kSmallFloats * sizeof(float) + 64;

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N = 256, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kH >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

// GELU in the tanh form of Hendrycks and Gimpel (2016),
//   0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))),
// with the hardware tanh approximation (tanh.approx.f32).  It departs from
// the erf form the network is trained with by at most 4.7e-4 (exact tanh),
// below the BF16 rounding of the activations the MMAs take; the erf form's
// library call was most of this kernel's time.
constexpr float kSqrt2OverPi = 0.7978845608028654f;
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float z) {
  const float u = kSqrt2OverPi * fmaf(0.044715f * z, z * z, z);
  return 0.5f * z * (1.f + tanh_approx(u));
}

// Byte offset of element (row r, k) of a K-major BF16 tile of 128-byte
// swizzle rows: chunk kc = k / 64 holds all rows' 128-byte segments, 8-row
// atoms of 1024 B, the 16-byte pieces of a row XOR-permuted by (row & 7).
__device__ __forceinline__ uint32_t act_offset(int r, int k) {
  const int kc = k >> 6, piece = (k & 63) >> 3;
  return (uint32_t)(kc * kActChunk + (r >> 3) * 1024 + (r & 7) * 128 + ((piece ^ (r & 7)) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// 8 consecutive activations (k0 multiple of 8) of row r as one 16-byte store.
__device__ __forceinline__ void store8(unsigned char* act, int r, int k0, const float (&v)[8]) {
  uint4 q;
  q.x = pack_bf16(v[0], v[1]);
  q.y = pack_bf16(v[2], v[3]);
  q.z = pack_bf16(v[4], v[5]);
  q.w = pack_bf16(v[6], v[7]);
  *reinterpret_cast<uint4*>(act + act_offset(r, k0)) = q;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int c = 0; c < 32; ++c) v[c] = __uint_as_float(r[c]);
}

// The 16 MMAs of one hidden layer: D[128 x 256] = A[128 x 256] * W^T, W^T
// K-major [256 x 256]; then a commit to `bar`.
__device__ __forceinline__ void layer_mma(uint32_t tmem, const unsigned char* act, const unsigned char* w,
                                          uint64_t* bar) {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
  for (int kc = 0; kc < kKChunks; ++kc) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint64_t ad = smem_desc_sw128(smem_u32(act + kc * kActChunk) + 32 * k);
      const uint64_t bd = smem_desc_sw128(smem_u32(w + kc * kWChunk) + 32 * k);
      const uint32_t acc = (kc | k) ? 1u : 0u;
      asm volatile(
          "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
          " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
          "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc));
    }
  }
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void load_weights(unsigned char* w, const CUtensorMap* map, uint64_t* bar) {
  mbar_expect_tx(bar, (uint32_t)kWBytes);
  for (int kc = 0; kc < kKChunks; ++kc) tma_load_2d(w + kc * kWChunk, map, kc * 64, 0, bar);
}

// FROM_X: features are the rows of x [n][8] and y [n] receives the network
// output; otherwise features come from the solver state (as mlp_features)
// and x0 [n] receives the guess 2 g_n - g_{n-1} + y.
template <bool FROM_X>
__global__ void __launch_bounds__(kRows, 1) mlp_tc_kernel(
    const __grid_constant__ CUtensorMap tmW2, const __grid_constant__ CUtensorMap tmW3, int n, const float* x,
    float* y_out, int num, int R, int C, const double* g_n, const double* g_nm1, const double* b_np1,
    const double* b_n, const double* phase, double* x0, const __nv_bfloat16* __restrict__ wbf,
    const float* __restrict__ master, size_t w1, size_t b1, size_t b2, size_t b3, size_t w4, size_t b4,
    const float* __restrict__ norm, int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char* act = base;            // [4][128][128 B] BF16 activations
  unsigned char* wt = act + kActBytes;  // [4][256][128 B] W^T of the current layer
  float* sW1 = reinterpret_cast<float*>(wt + kWBytes);  // [8][256]
  float* sB1 = sW1 + kMlpIn * kH;
  float* sB2 = sB1 + kH;
  float* sB3 = sB2 + kH;
  float* sW4 = sB3 + kH;
  uint64_t* bar_w = reinterpret_cast<uint64_t*>(sW4 + kH);
  uint64_t* bar_mma = bar_w + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_mma + 1);
  // thread 0 issues the copies and MMAs and does every mbarrier wait; the
  // outcome reaches the other threads through s_fail after a __syncthreads,
  // so that the warp-collective tcgen05.ld runs under a block-uniform branch
  __shared__ int s_fail, s_wpend, s_mpend;  // pending weight copy / MMA commit: 1 + its phase, 0 none
  const int tid = threadIdx.x, warp = tid >> 5;
  const int row0 = blockIdx.x * kRows;

  if (tid == 0) {
    s_fail = 0;
    s_wpend = s_mpend = 0;
    mbar_init(bar_w, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kH));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (tid == 0) {  // W2^T lands while layer 1 runs
    load_weights(wt, &tmW2, bar_w);
    s_wpend = 1;
  }
  // thread 0: bounded wait for `parity` of `bar`, failure into s_fail
  auto wait0 = [&](uint64_t* bar, uint32_t parity, int& pend) {
    if (s_fail) return;
    if (mbar_wait(bar, parity)) {
      pend = 0;
    } else {
      atomicExch(err, 1);
      s_fail = 1;
    }
  };

  // small operands into shared memory (FP32; W1 and w4 from their BF16 copies)
  for (int q = tid; q < kMlpIn * kH; q += kRows) sW1[q] = __bfloat162float(wbf[w1 + q]);
  for (int q = tid; q < kH; q += kRows) {
    sB1[q] = master[b1 + q];
    sB2[q] = master[b2 + q];
    sB3[q] = master[b3 + q];
    sW4[q] = __bfloat162float(wbf[w4 + q]);
  }
  __syncthreads();

  // 1. features of this thread's panel, normalised, and layer 1
  const int K = row0 + tid;
  float f[kMlpIn];
  if (K < n) {
    if (FROM_X) {
#pragma unroll
      for (int q = 0; q < kMlpIn; ++q) f[q] = x[(long long)K * kMlpIn + q];
    } else {
      const int per = R * C;
      const int wn = K / per, i = (K % per) / C, j = K % C;
      f[0] = (float)g_n[K];
      f[1] = (float)(g_n[K] - g_nm1[K]);
      f[2] = (float)b_np1[K];
      f[3] = (float)(b_np1[K] - b_n[K]);
      f[4] = (float)sin(phase[wn]);
      f[5] = (float)cos(phase[wn]);
      f[6] = 2.f * (i + 0.5f) / R - 1.f;
      f[7] = 2.f * (j + 0.5f) / C - 1.f;
    }
#pragma unroll
    for (int q = 0; q < kMlpIn; ++q) f[q] = (f[q] - norm[q]) / norm[kMlpIn + q];
  } else {
#pragma unroll
    for (int q = 0; q < kMlpIn; ++q) f[q] = 0.f;  // padding rows: computed, never stored
  }
#pragma unroll 1
  for (int c0 = 0; c0 < kH; c0 += 8) {
    float v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      float acc = 0.f;
#pragma unroll
      for (int q = 0; q < kMlpIn; ++q) acc = fmaf(f[q], sW1[q * kH + c0 + e], acc);
      v[e] = gelu(acc + sB1[c0 + e]);
    }
    store8(act, tid, c0, v);
  }
  // the generic-proxy stores must be visible to the tensor cores' reads
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  __syncthreads();

  // 2. layer 2; once its MMAs completed, W2^T and the layer-1 activations
  // are free: W3^T is brought over W2^T while the epilogue runs
  if (tid == 0) {
    wait0(bar_w, 0, s_wpend);
    if (!s_fail) {
      layer_mma(tmem, act, wt, bar_mma);
      s_mpend = 1;
      wait0(bar_mma, 0, s_mpend);
      if (!s_fail) {
        load_weights(wt, &tmW3, bar_w);
        s_wpend = 2;
      }
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
  if (!s_fail) {
#pragma unroll 1
    for (int j = 0; j < kH / 32; ++j) {
      float v[32];
      tmem_ld32(trow + (uint32_t)(j * 32), v);
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        float h[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) h[e] = gelu(v[g * 8 + e] + sB2[j * 32 + g * 8 + e]);
        store8(act, tid, j * 32 + g * 8, h);
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();

  // 3. layer 3
  if (tid == 0) {
    wait0(bar_w, 1, s_wpend);
    if (!s_fail) {
      layer_mma(tmem, act, wt, bar_mma);
      s_mpend = 2;
      wait0(bar_mma, 1, s_mpend);
    }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  // 4. head from TMEM
  if (!s_fail) {
    float acc = 0.f;
#pragma unroll 1
    for (int j = 0; j < kH / 32; ++j) {
      float v[32];
      tmem_ld32(trow + (uint32_t)(j * 32), v);
#pragma unroll
      for (int c = 0; c < 32; ++c) acc = fmaf(gelu(v[c] + sB3[j * 32 + c]), sW4[j * 32 + c], acc);
    }
    if (K < n) {
      const float y = (acc + master[b4]) * norm[2 * kMlpIn];
      if (FROM_X)
        y_out[K] = y;
      else
        x0[K] = 2.0 * g_n[K] - g_nm1[K] + (double)y;
    }
  }
  // after a timeout: wait (bounded) for this CTA's copies and MMAs in flight
  if (tid == 0) {
    if (s_wpend) mbar_wait(bar_w, (uint32_t)(s_wpend - 1));
    if (s_mpend) mbar_wait(bar_mma, (uint32_t)(s_mpend - 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kH));
}

// WT[c][k] = W[k][c] for the two hidden 256 x 256 layers (K-major B operands).
__global__ void transpose_hidden(const __nv_bfloat16* __restrict__ w, size_t off2, size_t off3,
                                 __nv_bfloat16* __restrict__ wT) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * kH * kH) return;
  const int l = q / (kH * kH), rem = q % (kH * kH), c = rem / kH, k = rem % kH;
  wT[q] = w[(l ? off3 : off2) + (size_t)k * kH + c];
}

}  // namespace

Error mlp_tc_set_wait_limit(long long cycles) { return set_wait_limit_here(cycles); }

bool mlp_tc_available() { return gemm_tc_available(); }

Error mlp_tc_prepare(Mlp* m, cudaStream_t st) {
  if (m->wT_version == m->version && m->wT) return ok();
  if (!load_encoder()) return fail(kErrUnsupported, "cuTensorMapEncodeTiled unavailable");
  if (!m->wT) UVLM_CUDA_TRY(cudaMalloc(&m->wT, sizeof(__nv_bfloat16) * 2 * kH * kH));
  if (!m->tc_err) {
    UVLM_CUDA_TRY(cudaMalloc(&m->tc_err, sizeof(int)));
    UVLM_CUDA_TRY(cudaMemset(m->tc_err, 0, sizeof(int)));
  }
  transpose_hidden<<<ceil_div(2 * kH * kH, 256), 256, 0, st>>>(m->wbf, m->layer[1].w_off, m->layer[2].w_off, m->wT);
  UVLM_LAUNCH_CHECK();
  for (int l = 0; l < 2; ++l)
    UVLM_TRY(encode_2d(&m->tmap[l], m->wT + (size_t)l * kH * kH, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, kH, kH,
                       (uint64_t)kH * 2, 64, kH));
  m->wT_version = m->version;
  return ok();
}

static Error launch_tc(Mlp* m, bool from_x, int n, const float* x, float* y, int num, int R, int C,
                       const double* g_n, const double* g_nm1, const double* b_np1, const double* b_n,
                       const double* phase, double* x0, cudaStream_t st) {
  if (n <= 0) return ok();
  UVLM_TRY(mlp_tc_prepare(m, st));
  auto kern = from_x ? mlp_tc_kernel<true> : mlp_tc_kernel<false>;
  UVLM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  const MlpLayer* L = m->layer;
  kern<<<ceil_div(n, kRows), kRows, kSmemBytes, st>>>(m->tmap[0], m->tmap[1], n, x, y, num, R, C, g_n, g_nm1, b_np1,
                                                      b_n, phase, x0, m->wbf, m->master, L[0].w_off, L[0].b_off,
                                                      L[1].b_off, L[2].b_off, L[3].w_off, L[3].b_off, m->norm,
                                                      m->tc_err);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error mlp_forward_tc(Mlp* m, const float* x, long long B, float* y, cudaStream_t st) {
  return launch_tc(m, true, (int)B, x, y, 0, 1, 1, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, st);
}

Error mlp_guess_tc(Mlp* m, int num, int R, int C, const double* g_n, const double* g_nm1, const double* b_np1,
                   const double* b_n, const double* phase, double* x0, cudaStream_t st) {
  return launch_tc(m, false, num * R * C, nullptr, nullptr, num, R, C, g_n, g_nm1, b_np1, b_n, phase, x0, st);
}

Error mlp_tc_check(Mlp* m, cudaStream_t st) {
  if (!m->tc_err) return ok();
  int h = 0;
  UVLM_CUDA_TRY(cudaMemcpyAsync(&h, m->tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  UVLM_CUDA_TRY(cudaStreamSynchronize(st));
  if (h) {
    UVLM_CUDA_TRY(cudaMemsetAsync(m->tc_err, 0, sizeof(int), st));
    return fail(kErrTimeout, "a bounded wait of the tensor-core MLP gave up");
  }
  return ok();
}

}  // namespace uvlm
