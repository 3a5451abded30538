// lu.cu -- blocked LU with partial pivoting, FP64 and FP32 factor types.
#include <climits>

#include <cooperative_groups.h>

#include "device_once.h"
#include "lu.cuh"

namespace uvlm {
namespace {

// Grid-wide barrier for cooperative launches.  bar[0] = arrival count,
// bar[1] = generation.  The wait is bounded: after g_wait_limit cycles the
// waiter sets err[0] (abort) and every CTA leaves at its next barrier.
__device__ bool grid_sync(unsigned* bar, unsigned nblocks, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = bar + 1;
    volatile int* verr = err;
    const unsigned g = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    int okv = 1;
    if (arrived == nblocks) {
      bar[0] = 0u;
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const long long t0 = clock64(), lim = g_wait_limit;
      while (*vgen == g) {
        if (verr[0]) { okv = 0; break; }
        if (clock64() - t0 > lim) { atomicExch(err, 1); okv = 0; break; }
        __nanosleep(32);
      }
    }
    __threadfence();
    if (verr[0]) okv = 0;
    s_ok = okv;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ inline void argmax_merge(double& v, int& r, double ov, int orow) {
  if (ov > v || (ov == v && orow < r)) { v = ov; r = orow; }
}

// Block-wide argmax of (|value|, row) with ties to the lower row.
__device__ void block_argmax(double& v, int& r) {
  __shared__ double sv[32];
  __shared__ int sr[32];
  for (int off = 16; off; off >>= 1) {
    const double ov = __shfl_down_sync(0xffffffffu, v, off);
    const int orow = __shfl_down_sync(0xffffffffu, r, off);
    argmax_merge(v, r, ov, orow);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { sv[wid] = v; sr[wid] = r; }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? sv[lane] : -1.0;
    r = lane < nw ? sr[lane] : INT_MAX;
    for (int off = 16; off; off >>= 1) {
      const double ov = __shfl_down_sync(0xffffffffu, v, off);
      const int orow = __shfl_down_sync(0xffffffffu, r, off);
      argmax_merge(v, r, ov, orow);
    }
    if (lane == 0) { sv[0] = v; sr[0] = r; }
  }
  __syncthreads();
  v = sv[0];
  r = sr[0];
  __syncthreads();
}

// One panel (columns k0..k0+kb-1, rows k0..n-1) of the factorisation.
// CTA b keeps panel rows [256 b, 256 b + 256) in shared memory, one row per
// thread (rows padded to kLuNB + 1 elements against bank conflicts).  Per
// column: block argmax of |a|, publish the CTA's candidate row (and the
// current diagonal row, by its owner), one grid barrier, every CTA picks the
// global pivot from the candidates, the two rows trade places and each thread
// eliminates its own row.
constexpr int kPanelRows = 256;
constexpr int kPanelLd = kLuNB + 1;

template <class T>
__global__ void __launch_bounds__(kPanelRows) lu_panel_kernel(T* A, int lda, int n, int k0, int kb, int* ipiv,
                                                              double* cand_val, int* cand_row, T* cand_data,
                                                              T* diag_data, unsigned* bar, int* err, int unused) {
  extern __shared__ __align__(16) unsigned char smraw[];
  T* rows = reinterpret_cast<T*>(smraw);         // [kPanelRows][kPanelLd]
  T* urow = rows + kPanelRows * kPanelLd;        // [kLuNB]
  __shared__ int s_piv, s_owner;
  (void)unused;
  const int P = gridDim.x, bid = blockIdx.x, tid = threadIdx.x;
  const int m = n - k0;
  const int rb = bid * kPanelRows;
  const int nloc = max(0, min(kPanelRows, m - rb));
  for (int q = tid; q < nloc * kb; q += blockDim.x) {
    const int r = q / kb, c = q % kb;
    rows[r * kPanelLd + c] = A[(long long)(k0 + rb + r) * lda + k0 + c];
  }
  __syncthreads();
  const bool mine = tid < nloc;
  T* my = rows + tid * kPanelLd;
  const int pr = rb + tid;  // this thread's panel row
  for (int c = 0; c < kb; ++c) {
    const int par = c & 1;
    double bv = -1.0;
    int br = INT_MAX;
    if (mine && pr >= c) {
      bv = fabs((double)my[c]);
      br = pr;
    }
    block_argmax(bv, br);
    if (tid == 0) {
      cand_val[par * kLuMaxCtas + bid] = bv;
      cand_row[par * kLuMaxCtas + bid] = (bv >= 0.0) ? br : -1;
    }
    if (bv >= 0.0)
      for (int q = tid; q < kb; q += blockDim.x)
        cand_data[((long long)par * kLuMaxCtas + bid) * kLuNB + q] = rows[(br - rb) * kPanelLd + q];
    if (c >= rb && c < rb + nloc)
      for (int q = tid; q < kb; q += blockDim.x) diag_data[par * kLuNB + q] = rows[(c - rb) * kPanelLd + q];
    __threadfence();
    if (!grid_sync(bar, (unsigned)P, err)) return;
    if (tid < 32) {
      double v = -1.0;
      int r = INT_MAX, ow = -1;
      for (int q = tid; q < P; q += 32) {
        const double cv = ((volatile double*)cand_val)[par * kLuMaxCtas + q];
        const int cr = ((volatile int*)cand_row)[par * kLuMaxCtas + q];
        if (cr >= 0 && (cv > v || (cv == v && cr < r))) { v = cv; r = cr; ow = q; }
      }
      for (int off = 16; off; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, v, off);
        const int orow = __shfl_down_sync(0xffffffffu, r, off);
        const int oow = __shfl_down_sync(0xffffffffu, ow, off);
        if (oow >= 0 && (ov > v || (ov == v && orow < r))) { v = ov; r = orow; ow = oow; }
      }
      if (tid == 0) {
        if (!(v > 0.0)) {  // zero column: record, do not swap
          atomicExch(err + 1, 1);
          r = c;
          ow = -1;
        }
        s_piv = r;
        s_owner = ow;
        if (bid == 0) ipiv[k0 + c] = k0 + r;
      }
    }
    __syncthreads();
    const int p = s_piv, ow = s_owner;
    const T* src = (ow >= 0) ? cand_data + ((long long)par * kLuMaxCtas + ow) * kLuNB : diag_data + par * kLuNB;
    for (int q = tid; q < kb; q += blockDim.x) urow[q] = ((volatile T*)src)[q];
    __syncthreads();
    // the pivot row's slot receives the old diagonal row; row c becomes the pivot row
    if (mine && pr == p && p != c)
      for (int q = 0; q < kb; ++q) my[q] = ((volatile T*)diag_data)[par * kLuNB + q];
    if (mine && pr == c)
      for (int q = 0; q < kb; ++q) my[q] = urow[q];
    if (mine && pr > c) {
      const T piv = urow[c];
      const T l = (piv != (T)0) ? my[c] / piv : (T)0;
      my[c] = l;
      for (int q = c + 1; q < kb; ++q) my[q] -= l * urow[q];
    }
    __syncthreads();
  }
  for (int q = tid; q < nloc * kb; q += blockDim.x) {
    const int r = q / kb, c = q % kb;
    A[(long long)(k0 + rb + r) * lda + k0 + c] = rows[r * kPanelLd + c];
  }
}

// The same panel factorisation for panels of at most kMaxClusterCtas x 256
// rows, as one thread-block cluster: the per-column pivot candidates, the
// pivot row and the displaced diagonal row are exchanged through distributed
// shared memory, and one hardware cluster barrier per column replaces the
// global-memory barrier.  Every CTA runs the same number of barriers.
constexpr int kMaxClusterCtas = 16;

template <class T>
__global__ void __launch_bounds__(kPanelRows) lu_panel_cluster_kernel(T* A, int lda, int n, int k0, int kb,
                                                                      int* ipiv, int* err) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smraw[];
  T* rows = reinterpret_cast<T*>(smraw);                     // [kPanelRows][kPanelLd]
  T* cand_data = rows + kPanelRows * kPanelLd;               // [2][kMaxClusterCtas][kLuNB]
  T* diag_data = cand_data + 2 * kMaxClusterCtas * kLuNB;    // [2][kLuNB]
  double* cand_val = reinterpret_cast<double*>(diag_data + 2 * kLuNB);  // [2][kMaxClusterCtas]
  int* cand_row = reinterpret_cast<int*>(cand_val + 2 * kMaxClusterCtas);  // [2][kMaxClusterCtas]
  __shared__ int s_piv, s_owner;
  const int P = (int)cl.num_blocks(), bid = (int)cl.block_rank(), tid = threadIdx.x;
  const int m = n - k0;
  const int rb = bid * kPanelRows;
  const int nloc = max(0, min(kPanelRows, m - rb));
  for (int q = tid; q < nloc * kb; q += blockDim.x) {
    const int r = q / kb, c = q % kb;
    rows[r * kPanelLd + c] = A[(long long)(k0 + rb + r) * lda + k0 + c];
  }
  __syncthreads();
  const bool mine = tid < nloc;
  T* my = rows + tid * kPanelLd;
  const int pr = rb + tid;
  for (int c = 0; c < kb; ++c) {
    const int par = c & 1;
    double bv = -1.0;
    int br = INT_MAX;
    if (mine && pr >= c) {
      bv = fabs((double)my[c]);
      br = pr;
    }
    block_argmax(bv, br);
    // Every CTA pushes its candidate (value, row, data) into slot `bid` of
    // every CTA's shared memory, and the CTA holding row c pushes that row;
    // after the cluster barrier each CTA reduces and swaps locally, so no
    // remote read follows the barrier.  A slot is rewritten two columns later
    // (double buffering), after the next barrier, when its readers are done.
    const bool has = bv >= 0.0;
    for (int idx = tid; idx < P * kb; idx += blockDim.x) {
      const int q = idx / kb, j = idx % kb;
      const T v = has ? rows[(br - rb) * kPanelLd + j] : (T)0;
      *cl.map_shared_rank(cand_data + (par * kMaxClusterCtas + bid) * kLuNB + j, q) = v;
    }
    if (tid < P) {
      *cl.map_shared_rank(cand_val + par * kMaxClusterCtas + bid, tid) = bv;
      *cl.map_shared_rank(cand_row + par * kMaxClusterCtas + bid, tid) = has ? br : -1;
    }
    if (c >= rb && c < rb + nloc)
      for (int idx = tid; idx < P * kb; idx += blockDim.x) {
        const int q = idx / kb, j = idx % kb;
        *cl.map_shared_rank(diag_data + par * kLuNB + j, q) = rows[(c - rb) * kPanelLd + j];
      }
    cl.sync();
    if (tid < 32) {
      double v = -1.0;
      int r = INT_MAX, ow = -1;
      for (int q = tid; q < P; q += 32) {
        const double cv = cand_val[par * kMaxClusterCtas + q];
        const int cr = cand_row[par * kMaxClusterCtas + q];
        if (cr >= 0 && (cv > v || (cv == v && cr < r))) { v = cv; r = cr; ow = q; }
      }
      for (int off = 16; off; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, v, off);
        const int orow = __shfl_down_sync(0xffffffffu, r, off);
        const int oow = __shfl_down_sync(0xffffffffu, ow, off);
        if (oow >= 0 && (ov > v || (ov == v && orow < r))) { v = ov; r = orow; ow = oow; }
      }
      if (tid == 0) {
        if (!(v > 0.0)) {
          atomicExch(err + 1, 1);
          r = c;
          ow = -1;
        }
        s_piv = r;
        s_owner = ow;
        if (bid == 0) ipiv[k0 + c] = k0 + r;
      }
    }
    __syncthreads();
    const int p = s_piv, ow = s_owner;
    const T* urow = (ow >= 0) ? cand_data + (par * kMaxClusterCtas + ow) * kLuNB : diag_data + par * kLuNB;
    const T* drow = diag_data + par * kLuNB;
    // the swap, each row copied by all threads of the CTA that holds it
    if (p != c && p >= rb && p < rb + nloc)
      for (int q = tid; q < kb; q += blockDim.x) rows[(p - rb) * kPanelLd + q] = drow[q];
    if (c >= rb && c < rb + nloc)
      for (int q = tid; q < kb; q += blockDim.x) rows[(c - rb) * kPanelLd + q] = urow[q];
    __syncthreads();
    if (mine && pr > c) {
      const T piv = urow[c];
      const T l = (piv != (T)0) ? my[c] / piv : (T)0;
      my[c] = l;
      for (int q = c + 1; q < kb; ++q) my[q] -= l * urow[q];
    }
    // the next column's block_argmax barrier orders these updates before
    // any thread reads another thread's row
  }
  cl.sync();
  for (int q = tid; q < nloc * kb; q += blockDim.x) {
    const int r = q / kb, c = q % kb;
    A[(long long)(k0 + rb + r) * lda + k0 + c] = rows[r * kPanelLd + c];
  }
}

// Launches the cluster panel kernel; false if the cluster cannot be formed
// (the caller then uses the cooperative kernel).
template <class T>
bool launch_panel_cluster(T* A, int n, int k0, int kb, int P, int* ipiv, int* err, cudaStream_t st) {
  if (P > kMaxClusterCtas) return false;
  auto kern = lu_panel_cluster_kernel<T>;
  const size_t smem = sizeof(T) * ((size_t)kPanelRows * kPanelLd + 2 * kMaxClusterCtas * kLuNB + 2 * kLuNB) +
                      2 * kMaxClusterCtas * (sizeof(double) + sizeof(int));
  // kernel attributes are per device: configure once on every device
  static PerDeviceOnce configured;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (!once_on_device(configured, dev, [&] {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
          cudaGetLastError();
          return false;
        }
        return true;
      }))
    return false;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P);
  cfg.blockDim = dim3(kPanelRows);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = P;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    return false;
  }
  if (cudaLaunchKernelEx(&cfg, kern, A, n, n, k0, kb, ipiv, err) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  note_launch();
  return true;
}

// ------------------------------------------------ tournament-pivoting panel
// The panel of kLuNB = 64 columns and m = n - k0 rows in one thread-block
// cluster of P = ceil(m / 256) CTAs (<= 16), with a few cluster barriers per
// panel instead of one per column.  The pivot rows are chosen by a tournament
// (communication-avoiding LU): each CTA factors its 256 rows with partial
// pivoting and keeps the 64 rows it picks, in pivot order; groups of up to
// four candidate sets are then merged by factoring their ORIGINAL rows
// (gathered from A, which the tournament does not modify) and keeping the 64
// rows picked, in a 4-ary tree over the cluster (the partners' lists are read
// through distributed shared memory).  The root's factorisation is the
// panel's top block L11\U11 in the root's pivot order.  The chosen rows are
// then brought to the top (LAPACK-style swap sequence in ipiv, replayed by
// every CTA for its own rows), and every other row r gets L21(r) from
// l U11 = a(r) (forward substitution on its original row).  The remaining
// columns are swapped by laswp and updated as before.  The pivots differ from
// column-by-column partial pivoting only where the candidates' magnitudes are
// close; the factorisation is of the same quality for the influence matrices
// of the path (and it backs a GMRES solve with FP64 residuals in the mixed
// form).
//
// Each factorisation keeps one row per thread in registers.  Column loop:
// blocks of 8 columns unrolled (compile-time register indices), a run-time
// loop over the blocks, and the row shifted left by 8 columns after each
// block (v[k] is column c0 + k), which keeps the code small and the row in
// registers.  Per column: a block argmax of (|a|, row id) packed into one
// 64-bit key (two warp max-reductions per level; ties go to the smaller row
// id, NaN counts as largest, a finished row has key 0 and never wins; for
// FP64 the 13 lowest mantissa bits make way for the id, so values within
// 2^-39 of each other count as tied); the pivot row's owner publishes its
// U part in shared memory; every other live row stores its multiplier in its
// shared-memory row of L (Lrow) and eliminates against the pivot row.  Two
// block barriers per column: a published row from one lane (one warp) costs
// less than every warp's candidate row before a single barrier.  Two lanes per
// row (16 warps, half rows, each lane reading half of the pivot row) measured
// 5 % (FP32) and 12 % (FP64) slower per panel than one lane per row.
constexpr int kTspRows = 256;  // rows per CTA = threads per CTA
constexpr int kTspMaxCtas = 16;
constexpr int kTspMaxRows = kTspRows * kTspMaxCtas;
constexpr int kTspLd = kLuNB + 1;  // Lrow stride: a column of Lrow is conflict-free
constexpr int kTspTop = kLuNB * kLuNB;

struct TspScratch {
  unsigned khi[2][kTspRows / 32];  // per-warp argmax keys, by step parity
  unsigned klo[2][kTspRows / 32];
  int list[kLuNB];    // this CTA's candidate ids (rows relative to k0), in pivot order
  int pivrow[kLuNB];  // the thread (Lrow row) of each pivot of the last factorisation
  int seq[kLuNB];     // the swap sequence (positions relative to k0)
  int cnt[4];         // [0] this CTA's candidate count; [1..3] partners' counts while merging
  short at[kTspMaxRows];   // original row (relative to k0) at each position
  short pos[kTspMaxRows];  // position of each original row
};

template <class T>
constexpr size_t tsp_smem() {
  return sizeof(T) * ((size_t)kTspTop + (size_t)kTspRows * kTspLd) + sizeof(TspScratch);
}

// One row of the panel (64 values from column k0) from A into registers;
// vector loads when the row start is 16-byte aligned.
template <class T>
__device__ __forceinline__ void tsp_load_row(const T* __restrict__ A, long long off, T (&v)[kLuNB]) {
  const T* src = A + off;
  if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    constexpr int kPer = 16 / sizeof(T);
#pragma unroll
    for (int q = 0; q < kLuNB / kPer; ++q) {
      if constexpr (sizeof(T) == 8) {
        const double2 t = reinterpret_cast<const double2*>(src)[q];
        v[2 * q] = t.x;
        v[2 * q + 1] = t.y;
      } else {
        const float4 t = reinterpret_cast<const float4*>(src)[q];
        v[4 * q] = t.x;
        v[4 * q + 1] = t.y;
        v[4 * q + 2] = t.z;
        v[4 * q + 3] = t.w;
      }
    }
  } else {
#pragma unroll
    for (int j = 0; j < kLuNB; ++j) v[j] = src[j];
  }
}

// Argmax key of a row: (hi, lo) compared lexicographically; 0 for a finished row.
template <class T>
__device__ __forceinline__ void tsp_key(T a, int id, bool alive, unsigned& hi, unsigned& lo) {
  hi = 0u;
  lo = 0u;
  if (!alive) return;
  const unsigned tag = 0x1000u - (unsigned)id;  // ids < 4096: 1 .. 0x1000, larger for smaller ids
  if constexpr (sizeof(T) == 4) {
    const float x = fabsf(a);
    hi = x != x ? 0xFFFFFFFFu : __float_as_uint(x);
    lo = tag;
  } else {
    const double x = fabs(a);
    const unsigned long long b = x != x ? ~0ull : (unsigned long long)__double_as_longlong(x);
    hi = (unsigned)(b >> 32);
    lo = ((unsigned)b & ~0x1FFFu) | tag;
  }
}

// Eight consecutive values at a 32-byte aligned address (vector accesses).
template <class T>
__device__ __forceinline__ void tsp_ld8(const T* p, T (&o)[8]) {
  if constexpr (sizeof(T) == 4) {
    const float4 a = reinterpret_cast<const float4*>(p)[0], b = reinterpret_cast<const float4*>(p)[1];
    o[0] = a.x, o[1] = a.y, o[2] = a.z, o[3] = a.w, o[4] = b.x, o[5] = b.y, o[6] = b.z, o[7] = b.w;
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double2 a = reinterpret_cast<const double2*>(p)[q];
      o[2 * q] = a.x;
      o[2 * q + 1] = a.y;
    }
  }
}

// uc[8 jc + t] = v[8 jc + t] (column c0 + 8 jc + t) for the 8-column chunks
// that reach column c (= c0 + k) and lie left of column 64 (the shifted row's
// entries past column 63 are dead); the chunk holding column c also writes
// the columns left of it, which no reader uses.
template <class T>
__device__ __forceinline__ void tsp_publish(T* uc, int c0, int k, const T (&v)[kLuNB]) {
#pragma unroll
  for (int jc = 0; jc < 8; ++jc) {
    if (8 * jc + 7 < k) continue;
    if (c0 + 8 * jc < kLuNB) {
      T* p = uc + 8 * jc;
      if constexpr (sizeof(T) == 4) {
        reinterpret_cast<float4*>(p)[0] = make_float4(v[8 * jc], v[8 * jc + 1], v[8 * jc + 2], v[8 * jc + 3]);
        reinterpret_cast<float4*>(p)[1] = make_float4(v[8 * jc + 4], v[8 * jc + 5], v[8 * jc + 6], v[8 * jc + 7]);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q)
          reinterpret_cast<double2*>(p)[q] = make_double2(v[8 * jc + 2 * q], v[8 * jc + 2 * q + 1]);
      }
    }
  }
}

// v[j] -= l uc[j] (column c0 + j of the pivot row) for the live columns
// j >= lo, chunk by chunk (chunks past column 63 hold dead entries of the
// shifted row and are skipped).
template <class T>
__device__ __forceinline__ void tsp_axpy(T (&v)[kLuNB], T l, const T* uc, int c0, int lo) {
#pragma unroll
  for (int jc = 0; jc < 8; ++jc) {
    if (8 * jc + 7 < lo) continue;
    if (c0 + 8 * jc < kLuNB) {
      T t8[8];
      tsp_ld8<T>(uc + 8 * jc, t8);
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (8 * jc + t >= lo) v[8 * jc + t] -= l * t8[t];
    }
  }
}

// The elimination of step c = c0 + k against the pivot row uc: l = v[k] /
// uc[k] into *lk, then v[j] -= l uc[j] for j > k.  A zero pivot leaves the
// row as it is and returns v[k] as its multiplier.
template <class T>
__device__ __forceinline__ void tsp_eliminate(T (&v)[kLuNB], const T* uc, int c0, int k, T* lk) {
  const T piv = uc[k];
  if (piv == (T)0) {
    *lk = v[k];
    return;
  }
  const T l = v[k] / piv;
  *lk = l;
  tsp_axpy<T>(v, l, uc, c0, k + 1);
}

template <class T>
__device__ __forceinline__ void tsp_shift8(T (&v)[kLuNB]) {
#pragma unroll
  for (int j = 0; j < kLuNB - 8; ++j) v[j] = v[j + 8];
}

// Partial-pivoting elimination of the R <= 256 rows held by threads
// 0 .. R-1 (v, original id myid).  Picks min(64, R) pivot rows: their ids go
// to out[] in pivot order, the owning threads to sc.pivrow[]; step c leaves
// the pivot row's U part in Top[c] (columns c .. 63) and every other row's
// multiplier in Lrow[thread][c].  Per column: the per-warp keys (of the
// step's parity: a slow reader of step c may still read them while a fast
// warp writes those of step c + 1) and a barrier; the block key; the owner
// publishes its row and a barrier; the others eliminate.  (Deferring all but
// the next column's update past the next argmax barrier measured 7-11 %
// slower per step; blocking by 8 columns with the update right of the block
// applied once per block measured the same as this.)  The operations on each row are those of a
// column-by-column factorisation, in the same order.  Every thread of the
// CTA calls it.
template <class T>
__device__ int tsp_factor(T (&v)[kLuNB], bool alive, int myid, int R, T* Top, T* Lrow, TspScratch& sc,
                          int* out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int steps = min(kLuNB, R);
  T* lrow = Lrow + tid * kTspLd;
#pragma unroll 1
  for (int c0 = 0; c0 < steps; c0 += 8) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int c = c0 + k;
      if (c < steps) {  // uniform
        const int par = c & 1;
        unsigned hi, lo;
        tsp_key<T>(v[k], myid, alive, hi, lo);
        const unsigned whi = __reduce_max_sync(0xffffffffu, hi);
        const unsigned wlo = __reduce_max_sync(0xffffffffu, hi == whi ? lo : 0u);
        if (lane == 0) {
          sc.khi[par][warp] = whi;
          sc.klo[par][warp] = wlo;
        }
        __syncthreads();
        const unsigned ph = lane < kTspRows / 32 ? sc.khi[par][lane] : 0u;
        const unsigned pl = lane < kTspRows / 32 ? sc.klo[par][lane] : 0u;
        const unsigned bhi = __reduce_max_sync(0xffffffffu, ph);
        const unsigned blo = __reduce_max_sync(0xffffffffu, ph == bhi ? pl : 0u);
        T* u = Top + c * kLuNB + c0;  // column c0 + j at u[j]
        if (alive && hi == bhi && lo == blo) {
          out[c] = 0x1000 - (int)(blo & 0x1FFFu);
          sc.pivrow[c] = tid;
          tsp_publish<T>(u, c0, k, v);
          alive = false;
        }
        __syncthreads();
        if (alive) tsp_eliminate<T>(v, u, c0, k, lrow + c);
      }
    }
    tsp_shift8<T>(v);
  }
  __syncthreads();  // Top, Lrow, out and pivrow complete for every thread
  return steps;
}

template <class T>
__global__ void __launch_bounds__(kTspRows, 1) lu_panel_tsp_kernel(T* A, int lda, int n, int k0, int* ipiv,
                                                                   int* err, int local) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smraw[];
  T* Top = reinterpret_cast<T*>(smraw);  // [64][64]: the pivot rows' U parts (columns c .. 63 of row c)
  T* Lrow = Top + kTspTop;               // [256][kTspLd]: multipliers of each thread's row
  TspScratch& sc = *reinterpret_cast<TspScratch*>(Lrow + kTspRows * kTspLd);
  const int P = (int)cl.num_blocks(), bid = (int)cl.block_rank(), tid = threadIdx.x;
  const int m = n - k0;
  const int rb = bid * kTspRows;
  const int nloc = max(0, min(kTspRows, m - rb));
  T v[kLuNB];

  // ---- phase 1: this CTA's rows (with local pivoting, only the first CTA's:
  // the pivots are chosen among the panel's top 256 rows)
  if (!local || bid == 0) {
    const bool alive = tid < nloc;
    if (alive) tsp_load_row<T>(A, (long long)(k0 + rb + tid) * lda + k0, v);
    const int k = tsp_factor<T>(v, alive, rb + tid, nloc, Top, Lrow, sc, sc.list);
    if (tid == 0) sc.cnt[0] = k;
  }

  // ---- phase 2: 4-ary tournament tree over the cluster; the merges factor
  // the candidates' original rows
  for (int step = 1; step < (local ? 1 : P); step *= 4) {
    cl.sync();  // the candidate lists of this level are final
    if ((bid % (4 * step)) == 0 && bid + step < P) {
      if (tid == 0)
        for (int g = 1; g < 4; ++g) {
          const int src = bid + g * step;
          sc.cnt[g] = src < P ? *cl.map_shared_rank(&sc.cnt[0], src) : 0;
        }
      __syncthreads();
      int R = 0, myid = INT_MAX;
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const int c = sc.cnt[g];
        if (tid >= R && tid < R + c)
          myid = g == 0 ? sc.list[tid - R] : *cl.map_shared_rank(&sc.list[tid - R], bid + g * step);
        R += c;
      }
      const bool alive = tid < R;
      if (alive) tsp_load_row<T>(A, (long long)(k0 + myid) * lda + k0, v);
      const int k = tsp_factor<T>(v, alive, myid, R, Top, Lrow, sc, sc.list);
      if (tid == 0) sc.cnt[0] = k;
    }
  }
  cl.sync();  // the root's Top, Lrow, pivrow and list are final

  // ---- phase 3: the swap sequence (CTA 0), sent to every CTA; the row map
  for (int q = tid; q < m; q += kTspRows) {
    sc.at[q] = (short)q;
    sc.pos[q] = (short)q;
  }
  __syncthreads();
  const int kb = kLuNB;  // m >= 64: the launcher's condition
  if (bid == 0 && tid == 0) {
    for (int i = 0; i < kb; ++i) {
      const int r = sc.list[i];
      const int qn = sc.pos[r];
      const int ri = sc.at[i];
      sc.at[i] = (short)r;
      sc.pos[r] = (short)i;
      sc.at[qn] = (short)ri;
      sc.pos[ri] = (short)qn;
      sc.seq[i] = qn;
      ipiv[k0 + i] = k0 + qn;
    }
  }
  __syncthreads();
  if (bid == 0)
    for (int q = tid; q < (P - 1) * kb; q += kTspRows) {
      const int c = 1 + q / kb, i = q - (c - 1) * kb;
      *cl.map_shared_rank(&sc.seq[i], c) = sc.seq[i];
    }
  cl.sync();
  if (bid > 0) {
    if (tid == 0)
      for (int i = 0; i < kb; ++i) {
        const int qn = sc.seq[i];
        const short t = sc.at[i];
        sc.at[i] = sc.at[qn];
        sc.at[qn] = t;
      }
    // U11 from the root
    const T* root = cl.map_shared_rank(Top, 0);
    for (int q = tid; q < kLuNB * kLuNB; q += kTspRows) Top[q] = root[q];
  }
  __syncthreads();
  // this CTA's rows below the top block: original values by new position
  const int p = rb + tid;
  const bool mine = tid < nloc && p >= kb;
  if (mine) tsp_load_row<T>(A, (long long)(k0 + sc.at[p]) * lda + k0, v);
  cl.sync();  // every CTA holds its original rows before any row of A is overwritten

  // ---- phase 4: the top block L11\U11 from the root, then L21 from l U11 = a
  if (bid == 0) {
    for (int q = tid; q < kb * kLuNB; q += kTspRows) {
      const int i = q / kLuNB, c = q - i * kLuNB;
      A[(long long)(k0 + i) * lda + k0 + c] = c < i ? Lrow[sc.pivrow[i] * kTspLd + c] : Top[q];
    }
    if (tid < kb && Top[tid * kLuNB + tid] == (T)0) atomicExch(err + 1, 1);
    __syncthreads();  // the root's Lrow is read before the substitution below overwrites it
  }
  if (mine) {
    // by columns: the operations, in order, of eliminating this row against
    // the pivot rows in a column-by-column factorisation
    T* lrow = Lrow + tid * kTspLd;
#pragma unroll 1
    for (int c0 = 0; c0 < kLuNB; c0 += 8) {
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int c = c0 + k;
        tsp_eliminate<T>(v, Top + c * kLuNB + c0, c0, k, lrow + c);
        if (Top[c * kLuNB + c] == (T)0) lrow[c] = (T)0;  // a zero pivot: multiplier 0 (the factor is singular)
      }
      tsp_shift8<T>(v);
    }
  }
  __syncthreads();
  for (int q = tid; q < nloc * kLuNB; q += kTspRows) {
    const int r = q >> 6, c = q & (kLuNB - 1);
    if (rb + r >= kb) A[(long long)(k0 + rb + r) * lda + k0 + c] = Lrow[r * kTspLd + c];
  }
  // every access to another CTA's shared memory came before the last cluster
  // barrier, so the CTAs may leave independently
}

// Launches the tournament panel; false when it cannot run (a panel narrower
// than 64 columns, too many rows for one cluster, or the cluster cannot be
// formed).
template <class T>
bool launch_panel_tsp(T* A, int n, int k0, int kb, int* ipiv, int* err, bool local, cudaStream_t st) {
  const int m = n - k0;
  const int P = ceil_div(m, kTspRows);
  if (P > kTspMaxCtas || kb != kLuNB || m < kLuNB) return false;
  auto kern = lu_panel_tsp_kernel<T>;
  const size_t smem = tsp_smem<T>();
  static PerDeviceOnce configured;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (!once_on_device(configured, dev, [&] {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
            cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
          cudaGetLastError();
          return false;
        }
        return true;
      }))
    return false;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(P);
  cfg.blockDim = dim3(kTspRows);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = P;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
    cudaGetLastError();
    return false;
  }
  if (cudaLaunchKernelEx(&cfg, kern, A, n, n, k0, ipiv, err, local ? 1 : 0) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  note_launch();
  return true;
}

// Row swaps of one panel applied to the columns outside the panel.
template <class T>
__global__ void laswp_kernel(T* A, int lda, int n, int k0, int kb, const int* __restrict__ ipiv) {
  const int other = n - kb;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < other; q += gridDim.x * blockDim.x) {
    const int col = q < k0 ? q : q + kb;
    for (int c = 0; c < kb; ++c) {
      const int p = ipiv[k0 + c];
      if (p != k0 + c) {
        T* a = A + (long long)(k0 + c) * lda + col;
        T* b = A + (long long)p * lda + col;
        const T t = *a;
        *a = *b;
        *b = t;
      }
    }
  }
}

// U12 = L11^-1 A12 (unit lower L11), one thread per column.  Optionally also
// writes U12 transposed into ut ([col - (k0+kb)][k], leading dim ldut).
// Columns per CTA of the TRSM (one column per thread; L11 staged once per
// CTA).  32-column CTAs, which spread a panel's columns over more SMs, took
// twice as long: each stages the whole L11 with a quarter of the threads.
constexpr int kTrsmThreads = 128;

template <class T>
__global__ void __launch_bounds__(kTrsmThreads) trsm_kernel(T* A, int lda, int n, int k0, int kb, T* ut, int ldut) {
  __shared__ T L[kLuNB][kLuNB + 1];
  if (kb == kLuNB) {
    // all of a thread's loads of L11 issued before any is stored (one round
    // trip, not one per element)
    constexpr int kPer = kLuNB * kLuNB / kTrsmThreads;
    T t[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int q = threadIdx.x + i * kTrsmThreads;
      t[i] = A[(long long)(k0 + q / kLuNB) * lda + k0 + q % kLuNB];
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int q = threadIdx.x + i * kTrsmThreads;
      L[q / kLuNB][q % kLuNB] = t[i];
    }
  } else {
    for (int q = threadIdx.x; q < kb * kb; q += blockDim.x) {
      const int r = q / kb, c = q % kb;
      L[r][c] = A[(long long)(k0 + r) * lda + k0 + c];
    }
  }
  __syncthreads();
  const int col = k0 + kb + blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  T x[kLuNB];
#pragma unroll
  for (int r = 0; r < kLuNB; ++r) x[r] = (r < kb) ? A[(long long)(k0 + r) * lda + col] : (T)0;
#pragma unroll
  for (int s = 0; s < kLuNB; ++s) {
#pragma unroll
    for (int r = s + 1; r < kLuNB; ++r) x[r] -= L[r][s] * x[s];
  }
#pragma unroll
  for (int r = 0; r < kLuNB; ++r)
    if (r < kb) A[(long long)(k0 + r) * lda + col] = x[r];
  if (ut) {
    T* o = ut + (long long)(col - k0 - kb) * ldut;
    bool done = false;
    if constexpr (sizeof(T) == 4) {
      if (kb == kLuNB && ldut % 4 == 0) {
        // whole rows of the transposed copy: 16-byte stores
#pragma unroll
        for (int r = 0; r < kLuNB; r += 4) *reinterpret_cast<float4*>(o + r) = make_float4(x[r], x[r + 1], x[r + 2], x[r + 3]);
        done = true;
      }
    }
    if (!done) {
#pragma unroll
      for (int r = 0; r < kLuNB; ++r)
        if (r < kb) o[r] = x[r];
    }
  }
}

// C -= A B with A [m x k] row-major (lda), B [k x nc] row-major (ldb).
template <class T>
__global__ void __launch_bounds__(256) gemm_update_kernel(T* C, int ldc, const T* __restrict__ A, int lda,
                                                          const T* __restrict__ B, int ldb, int m, int nc, int k) {
  constexpr int BM = 64, BN = 64, BK = 32;
  __shared__ __align__(16) T As[BK][BM];
  __shared__ __align__(16) T Bs[BK][BN];
  const int row0 = blockIdx.y * BM, col0 = blockIdx.x * BN;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = (T)0;
  for (int kk0 = 0; kk0 < k; kk0 += BK) {
    const int kc = min(BK, k - kk0);
    for (int q = tid; q < BM * BK; q += 256) {
      const int r = q / BK, kk = q % BK;
      As[kk][r] = (row0 + r < m && kk < kc) ? A[(long long)(row0 + r) * lda + kk0 + kk] : (T)0;
    }
    for (int q = tid; q < BK * BN; q += 256) {
      const int kk = q / BN, c = q % BN;
      Bs[kk][c] = (col0 + c < nc && kk < kc) ? B[(long long)(kk0 + kk) * ldb + col0 + c] : (T)0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < BK; ++kk) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = row0 + ty * 4 + i;
    if (r >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = col0 + tx * 4 + j;
      if (c < nc) C[(long long)r * ldc + c] -= acc[i][j];
    }
  }
}

// FP64 trailing update C -= A B of the plain form's LU (K = the panel width):
// 128 x 128 output tiles, 256 threads each holding an 8 x 8 register block
// (rows ty*4 + i and 64 + ty*4 + i, columns tx*4 + j and 64 + tx*4 + j), K
// in steps of 16 through a three-stage cp.async pipeline.  Each entry of C
// has its products subtracted one by one in k order (FMA), so the rounding
// differs from gemm_update_kernel's (which sums the products, then subtracts
// once) at the level of FP64 rounding.  The 16-byte copies need 16-byte
// aligned rows: even leading dimensions and aligned bases.
constexpr int kG64BM = 128, kG64BN = 128, kG64BK = 16, kG64Stages = 3;
constexpr int kG64ALd = kG64BK + 2;  // 144-byte rows of the A tile: the 4-row strides fall on other banks
constexpr int kG64StageA = kG64BM * kG64ALd;
constexpr int kG64StageB = kG64BK * kG64BN;
constexpr size_t kG64Smem = sizeof(double) * kG64Stages * (kG64StageA + kG64StageB);

__device__ __forceinline__ void cp_async16_zfill(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}

__global__ void __launch_bounds__(256, 1) gemm_update_f64_kernel(double* C, int ldc, const double* __restrict__ A,
                                                                 int lda, const double* __restrict__ B, int ldb,
                                                                 int m, int nc, int k) {
  extern __shared__ __align__(16) double g64_smem[];
  double* sA = g64_smem;                                // [stages][128][18]
  double* sB = g64_smem + kG64Stages * kG64StageA;     // [stages][16][128]
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int row0 = blockIdx.y * kG64BM, col0 = blockIdx.x * kG64BN;
  const int steps = (k + kG64BK - 1) / kG64BK;

  // 16-byte chunks (two doubles) of one K step; a chunk past the matrix is
  // zero-filled (the source address is then clamped to a valid one)
  auto load_step = [&](int t, int slot) {
    const int kk0 = t * kG64BK;
    double* a = sA + slot * kG64StageA;
    double* b = sB + slot * kG64StageB;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int q = tid + 256 * i;
      const int r = q >> 3, c2 = (q & 7) * 2;
      const int gr = row0 + r, gk = kk0 + c2;
      const int bytes = gr < m ? 8 * max(0, min(2, k - gk)) : 0;
      const double* src = bytes ? A + (long long)gr * lda + gk : A;
      cp_async16_zfill(a + r * kG64ALd + c2, src, bytes);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int q = tid + 256 * i;
      const int r = q >> 6, c2 = (q & 63) * 2;
      const int gk = kk0 + r, gc = col0 + c2;
      const int bytes = gk < k ? 8 * max(0, min(2, nc - gc)) : 0;
      const double* src = bytes ? B + (long long)gk * ldb + gc : B;
      cp_async16_zfill(b + r * kG64BN + c2, src, bytes);
    }
  };

  // the accumulators start as this thread's 8 x 8 block of C (loaded while
  // the operand pipeline fills) and the products are subtracted one by one,
  // so the tile's C traffic overlaps its loads instead of following the MMAs
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = row0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = col0 + h * 64 + tx * 4;
      const double* cp = C + (long long)r * ldc + c;
      if (r < m && c + 3 < nc) {
        const double2 v0 = *reinterpret_cast<const double2*>(cp);
        const double2 v1 = *reinterpret_cast<const double2*>(cp + 2);
        acc[i][h * 4 + 0] = v0.x;
        acc[i][h * 4 + 1] = v0.y;
        acc[i][h * 4 + 2] = v1.x;
        acc[i][h * 4 + 3] = v1.y;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][h * 4 + j] = (r < m && c + j < nc) ? cp[j] : 0.0;
      }
    }
  }

#pragma unroll
  for (int s = 0; s < kG64Stages - 1; ++s) {
    if (s < steps) load_step(s, s);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int t = 0; t < steps; ++t) {
    asm volatile("cp.async.wait_group %0;" ::"n"(kG64Stages - 2) : "memory");
    __syncthreads();  // step t landed for every thread; slot (t - 1) % stages is free
    if (t + kG64Stages - 1 < steps) load_step(t + kG64Stages - 1, (t + kG64Stages - 1) % kG64Stages);
    asm volatile("cp.async.commit_group;" ::: "memory");
    const double* a = sA + (t % kG64Stages) * kG64StageA;
    const double* b = sB + (t % kG64Stages) * kG64StageB;
#pragma unroll 8
    for (int kk = 0; kk < kG64BK; ++kk) {
      double av[8], bv[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        av[i] = a[(ty * 4 + i) * kG64ALd + kk];
        av[4 + i] = a[(64 + ty * 4 + i) * kG64ALd + kk];
      }
      const double2 b0 = *reinterpret_cast<const double2*>(b + kk * kG64BN + tx * 4);
      const double2 b1 = *reinterpret_cast<const double2*>(b + kk * kG64BN + tx * 4 + 2);
      const double2 b2 = *reinterpret_cast<const double2*>(b + kk * kG64BN + 64 + tx * 4);
      const double2 b3 = *reinterpret_cast<const double2*>(b + kk * kG64BN + 64 + tx * 4 + 2);
      bv[0] = b0.x, bv[1] = b0.y, bv[2] = b1.x, bv[3] = b1.y;
      bv[4] = b2.x, bv[5] = b2.y, bv[6] = b3.x, bv[7] = b3.y;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(-av[i], bv[j], acc[i][j]);
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");

#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = row0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
    if (r >= m) continue;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int c = col0 + h * 64 + tx * 4;
      double* cp = C + (long long)r * ldc + c;
      if (c + 3 < nc) {
        *reinterpret_cast<double2*>(cp) = make_double2(acc[i][h * 4 + 0], acc[i][h * 4 + 1]);
        *reinterpret_cast<double2*>(cp + 2) = make_double2(acc[i][h * 4 + 2], acc[i][h * 4 + 3]);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (c + j < nc) cp[j] = acc[i][h * 4 + j];
      }
    }
  }
}

// Inverses of the diagonal blocks: thread j < 64 forms column j of L_II^-1
// (unit lower), thread 64 + j column j of U_II^-1.
template <class T>
__global__ void diag_inverse_kernel(const T* LU, int n, T* dinv_l, T* dinv_u) {
  const int I = blockIdx.x;
  const int r0 = I * kTriB;
  const int nb = min(kTriB, n - r0);
  T* Li = dinv_l + (long long)I * kTriB * kTriB;
  T* Ui = dinv_u + (long long)I * kTriB * kTriB;
  const int j = threadIdx.x & (kTriB - 1);
  const bool upper = threadIdx.x >= kTriB;
  if (!upper) {
    for (int i = 0; i < kTriB; ++i) {
      T x = (i == j) ? (T)1 : (T)0;
      if (i < nb && j < nb && i > j) {
        for (int s = j; s < i; ++s) x -= LU[(long long)(r0 + i) * n + r0 + s] * Li[s * kTriB + j];
      }
      if (i >= nb || j >= nb) x = (i == j) ? (T)1 : (T)0;
      Li[i * kTriB + j] = (i < j) ? (T)0 : x;
    }
  } else {
    for (int i = kTriB - 1; i >= 0; --i) {
      T x = (T)0;
      if (i < nb && j < nb && i <= j) {
        x = (i == j) ? (T)1 : (T)0;
        for (int s = i + 1; s <= j; ++s) x -= LU[(long long)(r0 + i) * n + r0 + s] * Ui[s * kTriB + j];
        x = x / LU[(long long)(r0 + i) * n + r0 + i];
      } else if (i == j) {
        x = (T)1;
      }
      Ui[i * kTriB + j] = x;
    }
  }
}

// perm[k] = row of b that lands in row k after the LAPACK-style swap sequence.
__global__ void ipiv_to_perm_kernel(const int* ipiv, int n, int* perm) {
  // sp: the permutation, si: the pivot sequence (both staged by every thread;
  // the swaps themselves are one sequential chain in shared memory)
  extern __shared__ int sp[];
  int* si = sp + n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    sp[k] = k;
    si[k] = ipiv[k];
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < n; ++k) {
      const int p = si[k];
      const int t = sp[k];
      sp[k] = sp[p];
      sp[p] = t;
    }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) perm[k] = sp[k];
}

constexpr int kTriBatch = 8;  // block rows a CTA can consume in one pass

// Thread 0 waits (bounded) until the block row of solve-order position
// `first` is published, then counts how many of the following positions are
// published too (up to kTriBatch).  Returns that count, or 0 on abort.
__device__ int wait_ready(const unsigned* flags, int first, int left, bool lower, int nblk, unsigned epoch,
                          int* err) {
  __shared__ int s_cnt;
  if (threadIdx.x == 0) {
    const volatile unsigned* vf = flags;
    const int b0 = lower ? first : nblk - 1 - first;
    const long long t0 = clock64(), lim = g_wait_limit;
    int cnt = 1;
    while (vf[b0] != epoch) {
      if (((volatile int*)err)[0]) { cnt = 0; break; }
      if (clock64() - t0 > lim) { atomicExch(err + 2, 1); atomicExch(err, 1); cnt = 0; break; }
      __nanosleep(32);
    }
    if (cnt) {
      while (cnt < left && cnt < kTriBatch) {
        const int b = lower ? first + cnt : nblk - 1 - (first + cnt);
        if (vf[b] != epoch) break;
        ++cnt;
      }
    }
    __threadfence();
    s_cnt = cnt;
  }
  __syncthreads();
  return s_cnt;
}

// Sync-free blocked triangular solve.  lower: y = L^-1 (P v); upper: z = U^-1 y.
// CTA I owns block row I.  It consumes the block rows it depends on (J < I for
// the lower solve, J > I for the upper one) in solve order, taking in one pass
// every consecutive block row already published, so that once its last
// dependency appears only one 64x64 GEMV and the diagonal-inverse product
// remain on the critical path.  Each GEMV runs 4 threads per row with 16
// independent loads each.
template <class T, class V, bool kLower>
__global__ void __launch_bounds__(256) trsv_kernel(const T* __restrict__ LU, int n, const int* __restrict__ perm,
                                                   const double* __restrict__ vin, const V* yin, V* yout,
                                                   const T* __restrict__ dinv, unsigned* flags, unsigned epoch,
                                                   int* err, double* dout) {
  __shared__ V acc[kTriB];
  __shared__ V xs[kTriBatch * kTriB];
  const int nblk = gridDim.x;
  const int I = kLower ? blockIdx.x : nblk - 1 - blockIdx.x;
  const int r0 = I * kTriB;
  const int nb = min(kTriB, n - r0);
  const int tid = threadIdx.x;
  const int row = tid >> 2, quarter = tid & 3;
  if (tid < kTriB) {
    V v = 0;
    if (tid < nb) v = kLower ? (V)vin[perm[r0 + tid]] : yin[r0 + tid];
    acc[tid] = v;
  }
  __syncthreads();
  const int deps = kLower ? I : nblk - 1 - I;
  int done = 0;
  while (done < deps) {
    const int cnt = wait_ready(flags, done, deps - done, kLower, nblk, epoch, err);
    if (cnt == 0) return;
    for (int q = tid; q < cnt * kTriB; q += blockDim.x) {
      const int b = q / kTriB, c = q % kTriB;
      const int J = kLower ? done + b : nblk - 1 - (done + b);
      const int col = J * kTriB + c;
      xs[q] = (col < n) ? ((volatile V*)yout)[col] : (V)0;
    }
    __syncthreads();
    V s = 0;
    if (row < nb) {
      const T* rp = LU + (long long)(r0 + row) * n;
      for (int b = 0; b < cnt; ++b) {
        const int J = kLower ? done + b : nblk - 1 - (done + b);
        const int c0 = J * kTriB + quarter * 16;
        T a[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) a[c] = (c0 + c < n) ? rp[c0 + c] : (T)0;
#pragma unroll
        for (int c = 0; c < 16; ++c) s += (V)a[c] * xs[b * kTriB + quarter * 16 + c];
      }
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (quarter == 0 && row < nb) acc[row] -= s;
    __syncthreads();
    done += cnt;
  }
  // x_I = dinv_I * acc (4 threads per row)
  const T* D = dinv + (long long)I * kTriB * kTriB + (long long)row * kTriB + quarter * 16;
  V s = 0;
#pragma unroll
  for (int c = 0; c < 16; ++c) s += (V)D[c] * acc[quarter * 16 + c];
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  if (quarter == 0) xs[row] = s;
  __syncthreads();
  if (tid < nb) {
    yout[r0 + tid] = xs[tid];
    if (dout) dout[r0 + tid] = (double)xs[tid];
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) atomicExch(flags + I, epoch);
}

// Check of the bounded waits: one CTA waits, as a block row of the
// triangular solves waits for the rows before it, for a flag that nothing
// publishes; the wait must give up and report through err.
__global__ void wait_probe_kernel(const unsigned* flags, int* err) { wait_ready(flags, 0, 1, true, 1, 1u, err); }

template <class T>
Error lu_factor_impl(T* A, int n, LuUpdate upd, LuWork* w, cudaStream_t st) {
  if (n <= 0) return ok();
  if (n > kLuMaxCtas * kTriB) return fail(kErrUnsupported, "matrix larger than the cooperative solve supports");
  UVLM_CUDA_TRY(cudaMemsetAsync(w->err, 0, 4 * sizeof(int), st));
  UVLM_CUDA_TRY(cudaMemsetAsync(w->bar, 0, 2 * sizeof(unsigned), st));
  auto panel = lu_panel_kernel<T>;
  for (int k0 = 0; k0 < n; k0 += kLuNB) {
    const int kb = std::min(kLuNB, n - k0);
    const int m = n - k0;
    const int P = ceil_div(m, kPanelRows);
    if (P > std::min(w->num_sms, kLuMaxCtas)) return fail(kErrUnsupported, "matrix too large for the panel kernel");
    const int rpc = kPanelRows;
    size_t smem = sizeof(T) * ((size_t)kPanelRows * kPanelLd + kLuNB);
    if (smem > 48 * 1024) UVLM_CUDA_TRY(cudaFuncSetAttribute(panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int lda = n;
    int* ipiv = w->ipiv;
    double* cv = w->cand_val;
    int* cr = w->cand_row;
    T* cd = reinterpret_cast<T*>(w->cand_data);
    T* dd = reinterpret_cast<T*>(w->diag_data);
    unsigned* bar = w->bar;
    int* err = w->err;
    int nn = n, kk0 = k0, kkb = kb, rr = rpc;
    // tournament pivoting in one cluster; else the column-by-column cluster
    // panel; else the cooperative kernel
    if (!(w->tournament && launch_panel_tsp<T>(A, n, k0, kb, ipiv, err, w->local_pivot, st)) &&
        !launch_panel_cluster<T>(A, n, k0, kb, P, ipiv, err, st)) {
      void* args[] = {&A, &lda, &nn, &kk0, &kkb, &ipiv, &cv, &cr, &cd, &dd, &bar, &err, &rr};
      UVLM_CUDA_TRY(cudaLaunchCooperativeKernel((void*)panel, dim3(P), dim3(kPanelRows), args, smem, st));
      note_launch();
    }
    if (n - kb > 0) {
      const int other = n - kb;
      laswp_kernel<T><<<std::min(ceil_div(other, 256), 1024), 256, 0, st>>>(A, n, n, k0, kb, w->ipiv);
      UVLM_LAUNCH_CHECK();
    }
    const int rest = n - k0 - kb;
    if (rest > 0) {
      T* ut = (upd != kLuUpdateSimt) ? reinterpret_cast<T*>(w->ut) : nullptr;
      trsm_kernel<T><<<ceil_div(rest, kTrsmThreads), kTrsmThreads, 0, st>>>(A, n, n, k0, kb, ut, kLuNB);
      UVLM_LAUNCH_CHECK();
      T* C = A + (long long)(k0 + kb) * n + (k0 + kb);
      const T* L21 = A + (long long)(k0 + kb) * n + k0;
      const T* U12 = A + (long long)k0 * n + (k0 + kb);
      if constexpr (sizeof(T) == 8) {
        UVLM_TRY(gemm_update_f64(reinterpret_cast<double*>(C), n, reinterpret_cast<const double*>(L21), n,
                                 reinterpret_cast<const double*>(U12), n, rest, rest, kb, st));
      } else {
        // tensor-core update needs TMA-aligned rows (n % 4 == 0) and whole K chunks
        if (upd == kLuUpdateSimt || kb % 64 != 0 || n % 4 != 0) {
          UVLM_TRY(gemm_update_f32_simt(reinterpret_cast<float*>(C), n, reinterpret_cast<const float*>(L21), n,
                                        reinterpret_cast<const float*>(U12), n, rest, rest, kb, st));
        } else {
          UVLM_TRY(gemm_update_tc(reinterpret_cast<float*>(C), n, reinterpret_cast<const float*>(L21), n,
                                  reinterpret_cast<const float*>(w->ut), kLuNB, rest, rest, kb, upd, w, st));
        }
      }
    }
  }
  const int nblk = ceil_div(n, kTriB);
  diag_inverse_kernel<T><<<nblk, 2 * kTriB, 0, st>>>(A, n, reinterpret_cast<T*>(w->dinv_l),
                                                     reinterpret_cast<T*>(w->dinv_u));
  UVLM_LAUNCH_CHECK();
  // permutation vector stored after ipiv
  const size_t perm_smem = 2 * sizeof(int) * (size_t)n;
  if (perm_smem > 48 * 1024)
    UVLM_CUDA_TRY(cudaFuncSetAttribute(ipiv_to_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)perm_smem));
  ipiv_to_perm_kernel<<<1, 256, perm_smem, st>>>(w->ipiv, n, w->ipiv + n);
  UVLM_LAUNCH_CHECK();
  return ok();
}

template <class T, class V>
Error tri_solve(const T* LU, int n, LuWork* w, const double* vin, V* y, V* z, double* dout, cudaStream_t st) {
  const int nblk = ceil_div(n, kTriB);
  const unsigned epoch = ++w->epoch;
  const int* perm = w->ipiv + n;
  const T* dl = reinterpret_cast<const T*>(w->dinv_l);
  const T* du = reinterpret_cast<const T*>(w->dinv_u);
  unsigned* fl = w->flags;
  unsigned* fu = w->flags + kLuMaxCtas;
  int* err = w->err;
  double* nod = nullptr;
  const V* noy = nullptr;
  {
    auto k = trsv_kernel<T, V, true>;
    int nn = n;
    unsigned ep = epoch;
    void* args[] = {(void*)&LU, &nn, (void*)&perm, (void*)&vin, (void*)&noy, (void*)&y, (void*)&dl, &fl, &ep, &err, &nod};
    UVLM_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k, dim3(nblk), dim3(256), args, 0, st));
    note_launch();
  }
  {
    auto k = trsv_kernel<T, V, false>;
    int nn = n;
    unsigned ep = epoch;
    const V* yc = y;
    const double* nov = nullptr;
    void* args[] = {(void*)&LU, &nn, (void*)&perm, (void*)&nov, (void*)&yc, (void*)&z, (void*)&du, &fu, &ep, &err, &dout};
    UVLM_CUDA_TRY(cudaLaunchCooperativeKernel((void*)k, dim3(nblk), dim3(256), args, 0, st));
    note_launch();
  }
  return ok();
}

// Y = P (the row permutation of the factorisation as a dense matrix).
__global__ void identity_kernel(int n, float* Y) {
  const long long total = (long long)n * n;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(q / n), c = (int)(q % n);
    Y[q] = (c == r) ? 1.f : 0.f;
  }
}

// Y[rows r0 .. r0+nb) = D * Y[rows r0 .. r0+nb) on the columns below ncols,
// D a kTriB x kTriB block (rows/cols >= nb are identity padding), in place:
// each CTA owns 64 columns and reads its whole tile before writing.
__global__ void __launch_bounds__(256) apply_block_kernel(const float* __restrict__ D, float* Y, int n, int r0,
                                                          int nb, int ncols) {
  __shared__ float Ds[kTriB][kTriB + 1];
  __shared__ float Ts[kTriB][kTriB];
  const int c0 = blockIdx.x * 64;
  const int tid = threadIdx.x;
  for (int q = tid; q < kTriB * kTriB; q += 256) {
    const int i = q / kTriB, j = q % kTriB;
    Ds[i][j] = D[q];
    Ts[i][j] = (i < nb && c0 + j < ncols) ? Y[(long long)(r0 + i) * n + c0 + j] : 0.f;
  }
  __syncthreads();
  const int tx = tid & 15, ty = tid >> 4;
  float acc[4][4] = {};
  for (int s = 0; s < kTriB; ++s) {
    float a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = Ds[ty * 4 + i][s];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = Ts[s][tx * 4 + j];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = ty * 4 + i;
    if (r >= nb) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = c0 + tx * 4 + j;
      if (c < ncols) Y[(long long)(r0 + r) * n + c] = acc[i][j];
    }
  }
}

}  // namespace

// Split-TF32 operands of the inverse's rank-kTriB updates.  With hi(a) the
// TF32 rounding of a and lo(a) = a - hi(a) (exact in FP32), the update
//   C -= [hi(A) lo(A) hi(A)] [hi(B) hi(B) lo(B)]^T = A B - lo(A) lo(B)
// over K = 3 kTriB runs on the TF32 tensor cores with an error of the order
// of FP32 rounding, so the dense inverse is as accurate as FP32 triangular
// solves with the same factors.
__device__ __forceinline__ float tf32_hi(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return __uint_as_float(r);
}

// A3[i][0:64] = hi, [64:128] = lo, [128:192] = hi of A[i][0:64] (lda), i < m.
__global__ void split_a3_kernel(const float* __restrict__ A, int lda, int m, float* __restrict__ A3) {
  const long long total = (long long)m * kTriB;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const long long i = q / kTriB;
    const int k = (int)(q % kTriB);
    const float a = A[i * lda + k], h = tf32_hi(a);
    float* o = A3 + i * 3 * kTriB;
    o[k] = h;
    o[kTriB + k] = a - h;
    o[2 * kTriB + k] = h;
  }
}


namespace {
// apply_block_kernel and the B operand of the split-TF32 update in one pass,
// for a whole 64-row block: X[r0 .. r0+64) = D X[r0 .. r0+64) on the columns
// below ncols, written back, and its transposed split-TF32 copy
// B3[j][0:64] = hi, [64:128] = hi, [128:192] = lo of X[r0 + k][j] from the
// same values.  A CTA owns 32 columns: D and the X tile
// in shared memory, thread (k, group) forms the 8 products of row k for the
// group's 8 columns, then the tile goes out along rows of X and along k of B3.
__global__ void __launch_bounds__(256) apply_split_kernel(const float* __restrict__ D, float* X, int n, int r0,
                                                          int ncols, float* __restrict__ B3) {
  __shared__ float Ds[kTriB][kTriB + 1];
  __shared__ __align__(16) float Ts[kTriB][32];
  __shared__ float Ys[kTriB][33];
  const int j0 = blockIdx.x * 32;
  const int tid = threadIdx.x;
  {
    float dv[kTriB * kTriB / 256], tv[kTriB * 32 / 256];
#pragma unroll
    for (int u = 0; u < kTriB * kTriB / 256; ++u) dv[u] = D[tid + 256 * u];
#pragma unroll
    for (int u = 0; u < kTriB * 32 / 256; ++u) {
      const int q = tid + 256 * u, i = q >> 5, j = q & 31;
      tv[u] = j0 + j < ncols ? X[(long long)(r0 + i) * n + j0 + j] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kTriB * kTriB / 256; ++u) {
      const int q = tid + 256 * u;
      Ds[q / kTriB][q % kTriB] = dv[u];
    }
#pragma unroll
    for (int u = 0; u < kTriB * 32 / 256; ++u) {
      const int q = tid + 256 * u;
      Ts[q >> 5][q & 31] = tv[u];
    }
  }
  __syncthreads();
  const int k = tid & 63, g = tid >> 6;  // row k, columns 8 g .. 8 g + 7
  float acc[8] = {};
  for (int s = 0; s < kTriB; ++s) {
    const float a = Ds[k][s];
    const float4 b0 = *reinterpret_cast<const float4*>(&Ts[s][8 * g]);
    const float4 b1 = *reinterpret_cast<const float4*>(&Ts[s][8 * g + 4]);
    acc[0] += a * b0.x, acc[1] += a * b0.y, acc[2] += a * b0.z, acc[3] += a * b0.w;
    acc[4] += a * b1.x, acc[5] += a * b1.y, acc[6] += a * b1.z, acc[7] += a * b1.w;
  }
#pragma unroll
  for (int e = 0; e < 8; ++e) Ys[k][8 * g + e] = acc[e];
  __syncthreads();
  for (int q = tid; q < kTriB * 32; q += 256) {
    const int i = q >> 5, j = q & 31;
    if (j0 + j < ncols) X[(long long)(r0 + i) * n + j0 + j] = Ys[i][j];
  }
  for (int q = tid; q < kTriB * 32; q += 256) {
    const int j = q >> 6, kk = q & 63;
    if (j0 + j < ncols) {
      const float b = Ys[kk][j], h = tf32_hi(b);
      float* o = B3 + (long long)(j0 + j) * 3 * kTriB + kk;
      o[0] = h;
      o[kTriB] = h;
      o[2 * kTriB] = b - h;
    }
  }
}
}  // namespace

Error lu_inverse_f32(const float* LU, int n, LuUpdate upd, LuWork* w, float* X, cudaStream_t st) {
  if (n <= 0) return ok();
  const int nblk = ceil_div(n, kTriB);
  const float* dl = reinterpret_cast<const float*>(w->dinv_l);
  const float* du = reinterpret_cast<const float*>(w->dinv_u);
  identity_kernel<<<std::min<long long>(ceil_div((long long)n * n, 256), 4096), 256, 0, st>>>(n, X);
  UVLM_LAUNCH_CHECK();
  // Right-looking block substitution: each finished block row X_I (times the
  // inverse of its diagonal block) is subtracted from the rows still to come
  // in one rank-kTriB update, C -= A X_I, on the columns X_I can be non-zero
  // in: split-TF32 on the tensor cores when the operands are TMA-aligned
  // (n % 4 == 0, whole 64-row blocks), else SIMT.
  const bool tc = upd != kLuUpdateSimt && n % 4 == 0 && w->a3 != nullptr && w->b3 != nullptr;
  // X_I = D X_I (block row I, columns below ncols), then C -= A X_I; on the
  // tensor-core path the first two steps are one kernel that also writes X_I's
  // split-TF32 copy
  auto step = [&](const float* D, float* C, const float* A, int m, int ncols, int r0, int nb) -> Error {
    if (tc && nb == kTriB && m > 0) {
      apply_split_kernel<<<ceil_div(ncols, 32), 256, 0, st>>>(D, X, n, r0, ncols, w->b3);
      UVLM_LAUNCH_CHECK();
      split_a3_kernel<<<std::min<long long>(ceil_div((long long)m * kTriB, 256), 4096), 256, 0, st>>>(A, n, m, w->a3);
      UVLM_LAUNCH_CHECK();
      return gemm_update_tc(C, n, w->a3, 3 * kTriB, w->b3, 3 * kTriB, m, ncols, 3 * kTriB, kLuUpdateTF32, w, st);
    }
    apply_block_kernel<<<ceil_div(ncols, 64), 256, 0, st>>>(D, X, n, r0, nb, ncols);
    UVLM_LAUNCH_CHECK();
    if (m <= 0) return ok();
    return gemm_update_f32_simt(C, n, A, n, X + (long long)r0 * n, n, m, ncols, nb, st);
  };
  // X = L^-1 (L unit lower triangular, so X is too: block row I is non-zero
  // only in the columns below r1): X_I = Linv_II X_I, then
  // X_>I -= L_>I,I X_I on those columns
  for (int I = 0; I < nblk; ++I) {
    const int r0 = I * kTriB, nb = std::min(kTriB, n - r0), r1 = r0 + nb;
    UVLM_TRY(step(dl + (long long)I * kTriB * kTriB, X + (long long)r1 * n, LU + (long long)r1 * n + r0, n - r1, r1,
                  r0, nb));
  }
  // X = U^-1 X (dense): X_I = Uinv_II X_I, then X_<I -= U_<I,I X_I
  for (int I = nblk - 1; I >= 0; --I) {
    const int r0 = I * kTriB, nb = std::min(kTriB, n - r0);
    UVLM_TRY(step(du + (long long)I * kTriB * kTriB, X, LU + r0, r0, n, r0, nb));
  }
  return ok();
}

Error lu_work_alloc(LuWork* w, int n, int elem_size, int num_sms) {
  lu_work_free(w);
  w->n = n;
  w->elem_size = elem_size;
  w->num_sms = num_sms;
  const int nblk = ceil_div(n, kTriB);
  UVLM_CUDA_TRY(cudaMalloc(&w->ipiv, sizeof(int) * 2 * n));
  UVLM_CUDA_TRY(cudaMalloc(&w->err, sizeof(int) * 4));
  UVLM_CUDA_TRY(cudaMalloc(&w->bar, sizeof(unsigned) * 2));
  UVLM_CUDA_TRY(cudaMalloc(&w->cand_val, sizeof(double) * 2 * kLuMaxCtas));
  UVLM_CUDA_TRY(cudaMalloc(&w->cand_row, sizeof(int) * 2 * kLuMaxCtas));
  UVLM_CUDA_TRY(cudaMalloc(&w->cand_data, (size_t)elem_size * 2 * kLuMaxCtas * kLuNB));
  UVLM_CUDA_TRY(cudaMalloc(&w->diag_data, (size_t)elem_size * 2 * kLuNB));
  UVLM_CUDA_TRY(cudaMalloc(&w->dinv_l, (size_t)elem_size * nblk * kTriB * kTriB));
  UVLM_CUDA_TRY(cudaMalloc(&w->dinv_u, (size_t)elem_size * nblk * kTriB * kTriB));
  UVLM_CUDA_TRY(cudaMalloc(&w->flags, sizeof(unsigned) * 2 * kLuMaxCtas));
  UVLM_CUDA_TRY(cudaMemset(w->flags, 0, sizeof(unsigned) * 2 * kLuMaxCtas));
  UVLM_CUDA_TRY(cudaMemset(w->err, 0, sizeof(int) * 4));
  if (elem_size == 4) {
    UVLM_CUDA_TRY(cudaMalloc(&w->ut, sizeof(float) * (size_t)n * kLuNB));
    UVLM_CUDA_TRY(cudaMalloc(&w->a3, sizeof(float) * (size_t)n * 3 * kTriB));
    UVLM_CUDA_TRY(cudaMalloc(&w->b3, sizeof(float) * (size_t)n * 3 * kTriB));
    UVLM_CUDA_TRY(cudaMalloc(&w->opA, 2 * (size_t)n * kLuNB));
    UVLM_CUDA_TRY(cudaMalloc(&w->opB, 2 * (size_t)n * kLuNB));
  }
  w->epoch = 0;
  return ok();
}

void lu_work_free(LuWork* w) {
  cudaFree(w->ipiv);
  cudaFree(w->err);
  cudaFree(w->bar);
  cudaFree(w->cand_val);
  cudaFree(w->cand_row);
  cudaFree(w->cand_data);
  cudaFree(w->diag_data);
  cudaFree(w->dinv_l);
  cudaFree(w->dinv_u);
  cudaFree(w->flags);
  cudaFree(w->ut);
  cudaFree(w->a3);
  cudaFree(w->b3);
  cudaFree(w->opA);
  cudaFree(w->opB);
  *w = LuWork{};
}

Error lu_factor_f64(double* A, int n, LuWork* w, cudaStream_t st) {
  return lu_factor_impl<double>(A, n, kLuUpdateSimt, w, st);
}

Error lu_factor_f32(float* A, int n, LuUpdate upd, LuWork* w, cudaStream_t st) {
  return lu_factor_impl<float>(A, n, upd, w, st);
}

Error lu_check(LuWork* w, cudaStream_t st) {
  int h[4] = {0, 0, 0, 0};
  UVLM_CUDA_TRY(cudaMemcpyAsync(h, w->err, sizeof(h), cudaMemcpyDeviceToHost, st));
  UVLM_CUDA_TRY(cudaStreamSynchronize(st));
  if (h[0]) return fail(kErrTimeout, h[2] ? "triangular solve wait timed out" : "LU panel barrier timed out");
  if (h[1]) return fail(kErrSingular, "zero pivot in LU factorisation");
  return ok();
}

Error lu_solve_f64(const double* LU, int n, LuWork* w, const double* b, double* x, double* tmp, cudaStream_t st) {
  return tri_solve<double, double>(LU, n, w, b, tmp, x, nullptr, st);
}

Error lu_solve_f32(const float* LU, int n, LuWork* w, const double* v, double* z, float* tmp, cudaStream_t st) {
  return tri_solve<float, float>(LU, n, w, v, tmp, tmp + n, z, st);
}

Error gemm_update_f64(double* C, int ldc, const double* A, int lda, const double* B, int ldb, int m, int nc, int k,
                      cudaStream_t st) {
  if (m <= 0 || nc <= 0 || k <= 0) return ok();
  const bool aligned = lda % 2 == 0 && ldb % 2 == 0 && ldc % 2 == 0 &&
                       ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B) |
                         reinterpret_cast<uintptr_t>(C)) % 16) == 0;
  static PerDeviceOnce attr_once;
  int dev = 0;
  if (aligned && cudaGetDevice(&dev) == cudaSuccess && once_on_device(attr_once, dev, [] {
        return cudaFuncSetAttribute(gemm_update_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kG64Smem) == cudaSuccess;
      })) {
    dim3 grid(ceil_div(nc, kG64BN), ceil_div(m, kG64BM));
    gemm_update_f64_kernel<<<grid, 256, kG64Smem, st>>>(C, ldc, A, lda, B, ldb, m, nc, k);
    UVLM_LAUNCH_CHECK();
    return ok();
  }
  dim3 grid(ceil_div(nc, 64), ceil_div(m, 64));
  gemm_update_kernel<double><<<grid, 256, 0, st>>>(C, ldc, A, lda, B, ldb, m, nc, k);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error gemm_update_f32_simt(float* C, int ldc, const float* A, int lda, const float* B, int ldb, int m, int nc, int k,
                           cudaStream_t st) {
  if (m <= 0 || nc <= 0 || k <= 0) return ok();
  dim3 grid(ceil_div(nc, 64), ceil_div(m, 64));
  gemm_update_kernel<float><<<grid, 256, 0, st>>>(C, ldc, A, lda, B, ldb, m, nc, k);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error lu_set_wait_limit(long long cycles) { return set_wait_limit_here(cycles); }

Error lu_wait_probe(long long cycles, bool* gave_up) {
  unsigned* flags = nullptr;
  int* err = nullptr;
  UVLM_CUDA_TRY(cudaMalloc(&flags, 64 * sizeof(unsigned)));
  const cudaError_t e = cudaMalloc(&err, 4 * sizeof(int));
  if (e != cudaSuccess) {
    cudaFree(flags);
    return fail(kErrCuda, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  int h[4] = {0, 0, 0, 0};
  Error r = set_wait_limit_here(cycles);
  if (!r.code) {
    cudaMemset(flags, 0, 64 * sizeof(unsigned));
    cudaMemset(err, 0, 4 * sizeof(int));
    wait_probe_kernel<<<1, 64>>>(flags, err);
    note_launch();
    cudaError_t k = cudaGetLastError();
    if (k == cudaSuccess) k = cudaMemcpy(h, err, sizeof(h), cudaMemcpyDeviceToHost);
    if (k != cudaSuccess) r = fail(kErrCuda, std::string("wait probe: ") + cudaGetErrorString(k));
  }
  const Error restore = set_wait_limit_here(0);
  cudaFree(flags);
  cudaFree(err);
  if (r.code) return r;
  if (restore.code) return restore;
  *gave_up = h[0] != 0 && h[2] != 0;
  return ok();
}

}  // namespace uvlm
