// lu_tc.cu -- tcgen05 tensor-core trailing update of the mixed-precision LU:
//   C[m x nc] -= A[m x k] * Bt[nc x k]^T      (k = the panel width, 64)
// A is the L21 block of the factor (row-major, K-major for the MMA), Bt is
// U12 transposed by the TRSM (K-major as well).  One CTA per 128 x 128 output
// tile: TMA loads both operand tiles (128-byte swizzle) into shared memory,
// one thread issues the tcgen05.mma chain (kind::tf32 on the FP32 data, or
// kind::f16 on BF16 copies) accumulating in TMEM, and four warps read the
// accumulator with tcgen05.ld and subtract it from C along its rows (float4,
// staged through shared memory; C's loads are issued ahead, the first slice's
// before the MMAs, each next slice's before the current one is written).
// C's rows must be 16-byte aligned (C and ldc multiples of 4 floats), as the
// callers' TMA operands already require.  Every wait is bounded: on a timeout
// the CTA flags the error word, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "lu.cuh"
#include "tc_common.cuh"

namespace uvlm {
namespace {

constexpr int kBM = 128;
constexpr int kBN = 128;
constexpr int kRowBytes = 128;  // one swizzle row: 32 FP32 / 64 BF16 elements of K

// Instruction descriptor: FP32 accumulator, A/B format (2 = TF32, 1 = BF16),
// both K-major, N = kBN, M = kBM.
__host__ __device__ constexpr uint32_t make_idesc(uint32_t ab_format) {
  return (1u << 4) | (ab_format << 7) | (ab_format << 10) | ((uint32_t)(kBN >> 3) << 17) |
         ((uint32_t)(kBM >> 4) << 24);
}

// Loads one thread's share of a 32-column slice of C: rows row0 + 4 p
// (p < 8), the float4 at column col.  Rows past M and float4s that reach past
// N are left for the scalar tail path of the epilogue.
__device__ __forceinline__ void load_c_slice(const float* C, int ldc, int M, int N, int row0, int col,
                                             float4 (&cv)[8]) {
#pragma unroll
  for (int p = 0; p < 8; ++p) {
    const int row = row0 + p * 4;
    cv[p] = (row < M && col + 3 < N) ? *reinterpret_cast<const float4*>(C + (long long)row * ldc + col)
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

template <bool kBF16>
__global__ void __launch_bounds__(128, 1) tc_update_kernel(const __grid_constant__ CUtensorMap tmA,
                                                           const __grid_constant__ CUtensorMap tmB, int a_x0,
                                                           int a_y0, float* C, int ldc, int M, int N, int kchunks,
                                                           int* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  unsigned char* sA = base;                              // [kchunks][kBM][128 B]
  unsigned char* sB = sA + (size_t)kchunks * kBM * kRowBytes;  // [kchunks][kBN][128 B]
  uint64_t* bar_load = reinterpret_cast<uint64_t*>(sB + (size_t)kchunks * kBN * kRowBytes);
  uint64_t* bar_mma = bar_load + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar_mma + 1);
  __shared__ int s_fail;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;

  if (threadIdx.x == 0) {
    s_fail = 0;
    mbar_init(bar_load, 1);
    mbar_init(bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  // The epilogue's read of C does not depend on the MMAs: every thread issues
  // its loads of the first 32-column slice now, so that they overlap the
  // operand copies and the MMA chain (the loads of slice j + 1 overlap the
  // update of slice j below).
  const int sub = lane >> 3, q4 = (lane & 7) * 4;
  float4 cv[8];
  load_c_slice(C, ldc, M, N, m0 + warp * 32 + sub, n0 + q4, cv);

  if (threadIdx.x == 0) {
    const uint32_t bytes = (uint32_t)kchunks * (kBM + kBN) * kRowBytes;
    mbar_expect_tx(bar_load, bytes);
    constexpr int kElemsPerRow = kBF16 ? 64 : 32;
    for (int kc = 0; kc < kchunks; ++kc) {
      tma_load_2d(sA + (size_t)kc * kBM * kRowBytes, &tmA, a_x0 + kc * kElemsPerRow, a_y0 + m0, bar_load);
      tma_load_2d(sB + (size_t)kc * kBN * kRowBytes, &tmB, kc * kElemsPerRow, n0, bar_load);
    }
    if (!mbar_wait(bar_load, 0)) {
      atomicExch(err, 1);
      s_fail = 1;
    } else {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      constexpr uint32_t idesc = make_idesc(kBF16 ? 1u : 2u);
      // 4 MMAs per 128-byte row: K = 8 (TF32) or 16 (BF16) elements = 32 B each
      for (int kc = 0; kc < kchunks; ++kc) {
        for (int k = 0; k < 4; ++k) {
          const uint64_t ad = smem_desc_sw128(smem_u32(sA + (size_t)kc * kBM * kRowBytes) + 32 * k);
          const uint64_t bd = smem_desc_sw128(smem_u32(sB + (size_t)kc * kBN * kRowBytes) + 32 * k);
          const uint32_t acc = (kc | k) ? 1u : 0u;
          if (kBF16) {
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
          } else {
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(bar_mma))
                   : "memory");
    }
  }
  __syncthreads();
  bool ok = s_fail == 0;
  if (ok && !mbar_wait(bar_mma, 0)) {
    atomicExch(err, 1);
    ok = false;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    // Epilogue: each warp moves its 32 accumulator rows through a 32 x 33
    // shared-memory slice (4 x 4.2 KB inside the operand tiles, which are
    // free once the MMAs completed; at least 32 KB even for one K chunk) so
    // that the read-modify-write of C runs along rows: 8 lanes per row, a
    // float4 each, 4 rows per instruction.
    float* stage = reinterpret_cast<float*>(sA) + warp * 32 * 33;
#pragma unroll
    for (int j = 0; j < kBN / 32; ++j) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(j * 32);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
            "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
            "=r"(r[30]), "=r"(r[31])
          : "r"(taddr));
      float4 nx[8];
      if (j + 1 < kBN / 32) load_c_slice(C, ldc, M, N, m0 + warp * 32 + sub, n0 + (j + 1) * 32 + q4, nx);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int c = 0; c < 32; ++c) stage[lane * 33 + c] = __uint_as_float(r[c]);  // row = lane, column c
      __syncwarp();
      const int col = n0 + j * 32 + q4;
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const int rr = p * 4 + sub;
        const int row = m0 + warp * 32 + rr;
        const float* srow = stage + rr * 33 + q4;
        if (row < M) {
          float* c4 = C + (long long)row * ldc + col;
          if (col + 3 < N) {
            float4 v = cv[p];
            v.x -= srow[0];
            v.y -= srow[1];
            v.z -= srow[2];
            v.w -= srow[3];
            *reinterpret_cast<float4*>(c4) = v;
          } else {
            for (int e = 0; e < 4; ++e)
              if (col + e < N) c4[e] -= srow[e];
          }
        }
      }
      __syncwarp();
      if (j + 1 < kBN / 32) {
#pragma unroll
        for (int p = 0; p < 8; ++p) cv[p] = nx[p];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
}

// BF16 copies of the K-major operands (rows x 64, leading dim ld in floats).
__global__ void to_bf16_rows(const float* src, int ld, int rows, int k, __nv_bfloat16* dst) {
  const long long total = (long long)rows * k;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const long long r = q / k;
    const int c = (int)(q % k);
    dst[q] = __float2bfloat16(src[r * ld + c]);
  }
}

}  // namespace

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
}  // namespace

bool load_encoder() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  return g_encode != nullptr;
}

Error encode_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dt, int elem_bytes, uint64_t inner,
                uint64_t outer, uint64_t row_bytes, uint32_t box_inner, uint32_t box_outer) {
  const cuuint64_t dims[2] = {inner, outer};
  const cuuint64_t strides[1] = {row_bytes};
  const cuuint32_t box[2] = {box_inner, box_outer};
  const cuuint32_t estr[2] = {1, 1};
  (void)elem_bytes;
  const CUresult r = g_encode(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(kErrCuda, "cuTensorMapEncodeTiled failed");
  return ok();
}


Error tc_set_wait_limit(long long cycles) { return set_wait_limit_here(cycles); }

bool gemm_tc_available() {
  int dev = 0, major = 0, minor = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
  return major == 10 && minor == 0 && load_encoder();
}

Error gemm_update_tc(float* C, int ldc, const float* A, int lda, const float* Bt, int ldbt, int m, int nc, int k,
                     LuUpdate kind, LuWork* w, cudaStream_t st) {
  if (m <= 0 || nc <= 0) return ok();
  if (!load_encoder()) return fail(kErrUnsupported, "cuTensorMapEncodeTiled unavailable");
  // TMA: 16-byte aligned bases and row strides, inner coordinates on 128-byte rows
  if ((lda % 4) || (ldbt % 4) || (ldc % 4) || (k % (kind == kLuUpdateBF16 ? 64 : 32)) ||
      (reinterpret_cast<uintptr_t>(A) % 16) || (reinterpret_cast<uintptr_t>(Bt) % 16) ||
      (reinterpret_cast<uintptr_t>(C) % 16))
    return fail(kErrUnsupported, "operands not TMA-aligned");
  CUtensorMap ta, tb;
  int kchunks = 0, a_x0 = 0, a_y0 = 0;
  if (kind == kLuUpdateBF16) {
    auto* ab = reinterpret_cast<__nv_bfloat16*>(w->opA);
    auto* bb = reinterpret_cast<__nv_bfloat16*>(w->opB);
    to_bf16_rows<<<std::min(ceil_div((long long)m * k, 256), 8192), 256, 0, st>>>(A, lda, m, k, ab);
    UVLM_LAUNCH_CHECK();
    to_bf16_rows<<<std::min(ceil_div((long long)nc * k, 256), 8192), 256, 0, st>>>(Bt, ldbt, nc, k, bb);
    UVLM_LAUNCH_CHECK();
    UVLM_TRY(encode_2d(&ta, ab, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, k, m, (uint64_t)k * 2, 64, kBM));
    UVLM_TRY(encode_2d(&tb, bb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, k, nc, (uint64_t)k * 2, 64, kBN));
    kchunks = k / 64;
  } else {
    UVLM_TRY(encode_2d(&ta, A, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, k, m, (uint64_t)lda * 4, 32, kBM));
    UVLM_TRY(encode_2d(&tb, Bt, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, k, nc, (uint64_t)ldbt * 4, 32, kBN));
    kchunks = k / 32;
  }
  const size_t smem = 1024 + (size_t)kchunks * (kBM + kBN) * kRowBytes + 64;
  dim3 grid(ceil_div(nc, kBN), ceil_div(m, kBM));
  if (kind == kLuUpdateBF16) {
    auto kern = tc_update_kernel<true>;
    UVLM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, 128, smem, st>>>(ta, tb, a_x0, a_y0, C, ldc, m, nc, kchunks, w->err);
  } else {
    auto kern = tc_update_kernel<false>;
    UVLM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, 128, smem, st>>>(ta, tb, a_x0, a_y0, C, ldc, m, nc, kchunks, w->err);
  }
  UVLM_LAUNCH_CHECK();
  return ok();
}

}  // namespace uvlm
