// batch.cu -- many independent wings stepped together (uvlm_batch_*).
//
// Each case is one SimpleSimulator of a single wing (the reference runs one
// per process, simple_simulator.cpp:240-313); here every stage of
// MainLoop is ONE launch over all cases:
//   begin       G_prev <- G                                   (all rings)
//   kinematics  Morphing::Perfome of every node               (all nodes)
//   shed        TE node row (+ previous TE circulation row)   (all TE nodes)
//   geometry    collocation points, normals, areas, U_ls      (all rings)
//   assembly    A[K][L] = VORING(c_K, L, 1).n_K in FP64       (tile table)
//   rhs         wake N-body at the collocation points         (persistent)
//   solve       LU with partial pivoting, one CTA per case; mixed form: FP32
//               factors + FP64 iterative refinement with the FP64 matrix
//   loads       line N-body + Joukowski sums, one CTA per case
//   advect      wake N-body + Euler / RK2 update              (persistent)
// Sizes that grow with the wake (rows, targets, N-body work items) are derived
// on the device from a step counter, so the launch shapes never change and a
// whole step is captured once as a CUDA graph and replayed.
//
// Wake layout per case: a buffer of `cap` node rows; after the shed of step s
// the live node rows 0..s (0 = newest) sit at physical rows cap-1-s .. cap-1
// and ring row i at the same physical row as node row i (a prepend without a
// memmove, as SimpleSimulator::Shed prepends, simple_simulator.cpp:171-188).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/uvlm_b200.h"
#include "bs_math.cuh"
#include "host_lattice.h"
#include "nbody.cuh"
#include "step_math.cuh"

namespace uvlm {
namespace {

struct BCase {
  int R, C, N, lines;
  long long node_off, ring_off, line_off, mat_off;
  long long wnode_off, wring_off, wtgt_off, rec_off;
  double ff[3];
  double dt, area_ref;
  uvlm_kinematics kin;
};

// Prefix arrays (n + 1 entries) used to map a flat index to its case.
struct BPrefix {
  const long long* node;   // (R+1)(C+1)
  const long long* ring;   // R C
  const long long* line;   // R (2C+1)
  const long long* te;     // C+1
  const long long* rec;    // (R+1)(C+1) + cap (C+1)
  const long long* wnode;  // cap (C+1)
  const long long* wtgt;   // (cap-1)(C+1)
};

__device__ inline int find_case(const long long* pre, int n, long long g) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pre[mid] <= g)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__device__ inline WingShape shape_of(const BCase& b) { return WingShape{1, b.R, b.C}; }

// ------------------------------------------------------------ simple stages
// Start of a step: gamma_hist <- gamma_prev <- gamma (circulations of the
// last two steps; the loads need the last, the solve's extrapolated initial
// guess both).
__global__ void b_begin_kernel(const long long* __restrict__ ring_pre, int n, const double* gamma,
                               double* gamma_prev, double* gamma_hist) {
  const long long total = ring_pre[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    gamma_hist[g] = gamma_prev[g];
    gamma_prev[g] = gamma[g];
  }
}

__global__ void b_kinematics_kernel(const BCase* __restrict__ cs, BPrefix P, int n, const long long* d_step,
                                    const double* pos_init, double* pos) {
  const long long s = *d_step;
  const long long total = P.node[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const BCase& b = cs[find_case(P.node, n, g)];
    st3(pos + 3 * g, perfome(b.kin, ld3(pos_init + 3 * g), (double)s * b.dt));
  }
}

__global__ void b_shed_kernel(const BCase* __restrict__ cs, BPrefix P, int n, int cap, const long long* d_step,
                              const double* pos, const double* gamma, double* wpos, double* wgamma) {
  const long long s = *d_step;
  const long long total = P.te[n];
  const long long start = cap - 1 - s;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int c = find_case(P.te, n, g);
    const BCase& b = cs[c];
    const int j = (int)(g - P.te[c]);
    const double* p = pos + 3 * (b.node_off + (long long)b.R * (b.C + 1) + j);
    double* q = wpos + 3 * (b.wnode_off + start * (b.C + 1) + j);
    q[0] = p[0];
    q[1] = p[1];
    q[2] = p[2];
    if (s > 0 && j < b.C) wgamma[b.wring_off + start * b.C + j] = gamma[b.ring_off + (long long)(b.R - 1) * b.C + j];
  }
}

__global__ void b_geometry_kernel(const BCase* __restrict__ cs, BPrefix P, int n, const long long* d_step,
                                  const double* pos, const double* pos_init, double* cx, double* cy, double* cz,
                                  double* normal, double* area, double* uls) {
  const long long s = *d_step;
  const long long total = P.ring[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const BCase& b = cs[find_case(P.ring, n, g)];
    const WingShape ws = shape_of(b);
    const int K = (int)(g - b.ring_off);
    const int i = K / b.C, j = K % b.C;
    const double* ps = pos + 3 * b.node_off;
    const double* p0 = pos_init + 3 * b.node_off;
    const d3 p00 = ld3(ps + 3 * ws.node(0, i, j)), p10 = ld3(ps + 3 * ws.node(0, i + 1, j));
    const d3 p11 = ld3(ps + 3 * ws.node(0, i + 1, j + 1)), p01 = ld3(ps + 3 * ws.node(0, i, j + 1));
    const d3 c = dvs(add(add(add(p00, p10), p11), p01), 4);  // simple_simulator.cpp:19-32
    cx[g] = c.x;
    cy[g] = c.y;
    cz[g] = c.z;
    st3(normal + 3 * g, normalized(cross(sub(p11, p00), sub(p01, p10))));  // :34-50
    area[g] = norm(cross(sub(p10, p00), sub(p01, p00)));                   // joukowski.cpp:55-67
    const d3 q00 = ld3(p0 + 3 * ws.node(0, i, j)), q10 = ld3(p0 + 3 * ws.node(0, i + 1, j));
    const d3 q11 = ld3(p0 + 3 * ws.node(0, i + 1, j + 1)), q01 = ld3(p0 + 3 * ws.node(0, i, j + 1));
    st3(uls + 3 * g, morph_velocity(b.kin, dvs(add(add(add(q00, q10), q11), q01), 4), (double)s * b.dt));
  }
}

// ---------------------------------------------------------------- assembly
// FP64 influence matrix of every case by unique lattice segments, as the
// single-case assembly: one lane per (collocation point K, node column j)
// walks the node rows and writes ring (i-1, j) = S(i-1, j) + H(i-1, j+1) -
// S(i, j) - H(i-1, j) (VORING's p0 -> p1 -> p2 -> p3 -> p0, src/vortex.cpp:145-160),
// H(i-1, j+1) from the next lane; warps advance 31 positions.  Tile = (case,
// a range [p0, p1) of its (K, node column) positions, K-major).
struct AsmTile {
  int c;
  long long p0, p1;
};
constexpr int kBAsmThreads = 128;
constexpr int kBAsmPerWarp = 31;
constexpr int kBAsmTilePositions = kBAsmPerWarp * (kBAsmThreads / 32) * 8;

__global__ void __launch_bounds__(kBAsmThreads) b_assemble_kernel(const BCase* __restrict__ cs,
                                                                  const AsmTile* __restrict__ tiles,
                                                                  const double* __restrict__ pos,
                                                                  const double* __restrict__ cx,
                                                                  const double* __restrict__ cy,
                                                                  const double* __restrict__ cz,
                                                                  const double* __restrict__ normal, double* A) {
  const AsmTile T = tiles[blockIdx.x];
  const BCase& b = cs[T.c];
  const WingShape ws = shape_of(b);
  const int C1 = b.C + 1;
  const long long P = (long long)b.N * C1;
  const int lane = threadIdx.x & 31;
  const double* ps = pos + 3 * b.node_off;
  const double g = 1.0 / (4.0 * kPi);
  double* Ac = A + b.mat_off;
  for (long long base = T.p0 + (long long)(threadIdx.x >> 5) * kBAsmPerWarp; base < T.p1;
       base += (long long)kBAsmPerWarp * (kBAsmThreads / 32)) {
    // the halo lane may read the position after the tile (or the case's last again)
    const long long p = min(base + lane, P - 1);
    const int K = (int)(p / C1), j = (int)(p - (long long)K * C1);
    const bool owner = lane < kBAsmPerWarp && base + lane < T.p1 && j < b.C;
    const int j1 = min(j + 1, b.C);
    const long long Kg = b.ring_off + K;
    const double X = cx[Kg], Y = cy[Kg], Z = cz[Kg];
    const double nx = normal[3 * Kg], ny = normal[3 * Kg + 1], nz = normal[3 * Kg + 2];
    auto node_at = [&](int i, int jj) {
      const double* q = ps + 3 * ws.node(0, i, jj);
      return make_node<double>(X - q[0], Y - q[1], Z - q[2]);
    };
    Node<double> na = node_at(0, j), nb = node_at(0, j1);
    double sx = 0, sy = 0, sz = 0;  // S(i-1, j)
    segment<double>(na, nb, g, sx, sy, sz);
    double* row = Ac + (long long)K * b.N + j;
    for (int i = 1; i <= b.R; ++i) {
      const Node<double> na2 = node_at(i, j), nb2 = node_at(i, j1);
      double hx = 0, hy = 0, hz = 0;  // H(i-1, j)
      segment<double>(na, na2, g, hx, hy, hz);
      const double hnx = __shfl_down_sync(0xffffffffu, hx, 1);  // H(i-1, j+1)
      const double hny = __shfl_down_sync(0xffffffffu, hy, 1);
      const double hnz = __shfl_down_sync(0xffffffffu, hz, 1);
      double s2x = 0, s2y = 0, s2z = 0;  // S(i, j)
      segment<double>(na2, nb2, g, s2x, s2y, s2z);
      if (owner) {
        const double vx = ((sx + hnx) - s2x) - hx;
        const double vy = ((sy + hny) - s2y) - hy;
        const double vz = ((sz + hnz) - s2z) - hz;
        row[(long long)(i - 1) * b.C] = vx * nx + vy * ny + vz * nz;
      }
      na = na2;
      nb = nb2;
      sx = s2x;
      sy = s2y;
      sz = s2z;
    }
  }
}

// ------------------------------------------------------- N-body plumbing
enum BStage { kStageRhs = 0, kStageLoads = 1, kStageAdvect = 2 };

// Source records of every case: [bound sheet (R+1)(C+1)][wake sheet, node
// rows 0..s from `wsrc`]; with_bound = 0 rewrites only the wake part.
template <class Rec>
__global__ void b_records_kernel(const BCase* __restrict__ cs, BPrefix P, int n, int cap, const long long* d_step,
                                 int with_bound, const double* pos, const double* gamma, const double* wsrc,
                                 const double* wgamma, Rec* rec) {
  const long long s = *d_step;
  const long long total = P.rec[n];
  const int start = (int)(cap - 1 - s);
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int c = find_case(P.rec, n, g);
    const BCase& b = cs[c];
    const long long k = g - P.rec[c];
    const long long nb = (long long)(b.R + 1) * (b.C + 1);
    if (k < nb) {
      if (!with_bound) continue;
      SheetView v{pos + 3 * b.node_off, b.R + 1, 0, gamma + b.ring_off, b.R, 0, 1, b.R + 1, b.C};
      rec[b.rec_off + k] = build_record<Rec>(v, k);
    } else {
      const long long kw = k - nb;
      if (kw >= (s + 1) * (b.C + 1)) continue;
      SheetView v{wsrc + 3 * b.wnode_off, cap, start, wgamma + b.wring_off, cap, start, 1, (int)(s + 1), b.C};
      rec[b.rec_off + nb + kw] = build_record<Rec>(v, kw);
    }
  }
}

__global__ void b_nbody_inputs_kernel(const BCase* __restrict__ cs, int n, const long long* d_step, int stage,
                                      NBodyBatchInput* in) {
  const long long s = *d_step;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const BCase& b = cs[c];
    NBodyBatchInput x{};
    const long long nb = (long long)(b.R + 1) * (b.C + 1);
    const SourceBlock wake{b.rec_off + nb, 1, (int)(s + 1), b.C};
    if (stage == kStageRhs) {
      x.blocks[0] = wake;
      x.n_blocks = 1;
      x.tgt_off = b.ring_off;
      x.n_tgt = b.N;
    } else {
      x.blocks[0] = SourceBlock{b.rec_off, 1, b.R + 1, b.C};
      x.blocks[1] = wake;
      x.n_blocks = 2;
      if (stage == kStageLoads) {
        x.tgt_off = b.line_off;
        x.n_tgt = b.lines;
      } else {
        x.tgt_off = b.wtgt_off;
        x.n_tgt = s * (b.C + 1);  // wake node rows 1..s (row 0 moves with -ff)
      }
    }
    in[c] = x;
  }
}

// b_K = -(Uw - (Uls + ff)) . n_K (simple_simulator.cpp:103-124)
__global__ void b_rhs_kernel(const BCase* __restrict__ cs, BPrefix P, int n, const double* vx, const double* vy,
                             const double* vz, const double* uls, const double* normal, double* rhs) {
  const long long total = P.ring[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const BCase& b = cs[find_case(P.ring, n, g)];
    const d3 u = sub(mk(vx[g], vy[g], vz[g]), add(ld3(uls + 3 * g), mk(b.ff[0], b.ff[1], b.ff[2])));
    rhs[g] = -dot(u, ld3(normal + 3 * g));
  }
}

// ------------------------------------------------------------- dense solve
// Threads of the per-case solve CTA: the FP32-factor form (refinement sweeps,
// latency-bound streaming on the largest cases) takes 16 warps; the FP64
// form, which factors every step, 8 (its panel code keeps its registers).
template <class T>
struct SolveCfg {
  static constexpr int kThreads = sizeof(T) == 4 ? 512 : 256;
};

// Panel width of the shared-memory LU: 32 FP32 / 16 FP64 columns, so that
// the whole panel of the largest case (1024 rows) stays in shared memory.
template <class T>
struct PanelCfg {
  static constexpr int NB = sizeof(T) == 4 ? 32 : 16;
  static constexpr int LD = NB + 1;  // padded row (conflict-free column walks)
};

inline size_t panel_smem_bytes(int max_N, int elem) {
  const int nb = elem == 4 ? 32 : 16;
  return (size_t)max_N * (nb + 1) * elem;
}

// Right-looking blocked LU with partial pivoting of the row-major N x N
// matrix A by one CTA.  Each panel of NB columns is held in shared memory
// while it is factored (the pivot of column j is the largest |a| at or below
// the diagonal, ties to the lower index; pivot search, swaps, scaling and the
// rank-1 updates walk shared memory instead of strided rows in L2).  The
// panel's row swaps are then applied to the other columns (LAPACK order),
// U12 = L11^-1 A12 is solved column per thread with L11 from shared memory,
// and A22 -= L21 U12 reads L21 from shared memory.  piv[j] = row swapped
// with j.  P: (N - k0) x LD panel buffer in dynamic shared memory.
template <class T>
__device__ void cta_lu_panel_smem(T* A, int N, int* piv, int* status, T* P) {
  constexpr int NB = PanelCfg<T>::NB, LD = PanelCfg<T>::LD;
  constexpr int NT = SolveCfg<T>::kThreads;
  constexpr int TR = NT / 16 * 4;  // rows of an A22 tile (16 threads x 4 columns across, 4 rows each)
  __shared__ double s_val[NT / 32];
  __shared__ int s_idx[NT / 32];
  __shared__ int s_piv[NB];
  __shared__ T Bs[NB][64];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int k0 = 0; k0 < N; k0 += NB) {
    const int kb = min(NB, N - k0);
    const int m = N - k0;
    for (int q = tid; q < m * NB; q += NT) {
      const int r = q / NB, c = q % NB;
      P[r * LD + c] = c < kb ? A[(long long)(k0 + r) * N + k0 + c] : (T)0;
    }
    __syncthreads();
    for (int jj = 0; jj < kb; ++jj) {
      double best = -1.0;
      int bi = jj;
      for (int i = jj + tid; i < m; i += NT) {
        const double v = fabs((double)P[i * LD + jj]);
        if (v > best) {
          best = v;
          bi = i;
        }
      }
      for (int off = 16; off; off >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, best, off);
        const int oi = __shfl_down_sync(0xffffffffu, bi, off);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
        }
      }
      if (lane == 0) {
        s_val[wid] = best;
        s_idx[wid] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        double bv = s_val[0];
        int ii = s_idx[0];
        for (int w = 1; w < NT / 32; ++w)
          if (s_val[w] > bv || (s_val[w] == bv && s_idx[w] < ii)) {
            bv = s_val[w];
            ii = s_idx[w];
          }
        s_piv[jj] = ii;
        piv[k0 + jj] = k0 + ii;
        if (!(bv > 0)) status[1] = 1;
      }
      __syncthreads();
      const int p = s_piv[jj];
      if (p != jj && tid < NB) {
        const T t = P[jj * LD + tid];
        P[jj * LD + tid] = P[p * LD + tid];
        P[p * LD + tid] = t;
      }
      __syncthreads();
      const T d = P[jj * LD + jj];
      for (int i = jj + 1 + tid; i < m; i += NT) {
        T* row = P + i * LD;
        const T l = row[jj] / d;
        row[jj] = l;
        for (int c = jj + 1; c < kb; ++c) row[c] -= l * P[jj * LD + c];
      }
      __syncthreads();
    }
    // panel back to global memory
    for (int q = tid; q < m * NB; q += NT) {
      const int r = q / NB, c = q % NB;
      if (c < kb) A[(long long)(k0 + r) * N + k0 + c] = P[r * LD + c];
    }
    // the panel's swaps on the columns left and right of it, in order
    for (int jj = 0; jj < kb; ++jj) {
      const int p = s_piv[jj];
      if (p != jj) {
        T* ra = A + (long long)(k0 + jj) * N;
        T* rb = A + (long long)(k0 + p) * N;
        for (int c = tid; c < N - kb; c += NT) {
          const int col = c < k0 ? c : c + kb;
          const T t = ra[col];
          ra[col] = rb[col];
          rb[col] = t;
        }
      }
      __syncthreads();
    }
    const int c0 = k0 + kb;
    if (c0 >= N) break;
    // U12 = L11^-1 A12: column per thread, the column in registers
    for (int c = c0 + tid; c < N; c += NT) {
      T u[NB];
#pragma unroll
      for (int i = 0; i < NB; ++i) u[i] = i < kb ? A[(long long)(k0 + i) * N + c] : (T)0;
#pragma unroll
      for (int i = 1; i < NB; ++i) {
        T s = u[i];
#pragma unroll
        for (int l = 0; l < i; ++l) s -= P[i * LD + l] * u[l];
        u[i] = s;
      }
#pragma unroll
      for (int i = 1; i < NB; ++i)
        if (i < kb) A[(long long)(k0 + i) * N + c] = u[i];
    }
    __syncthreads();
    // A22 -= L21 U12 in TR x 64 tiles, L21 = panel rows kb.. (shared memory)
    const int mt = N - c0;
    const int rtiles = (mt + TR - 1) / TR, ctiles = (mt + 63) / 64;
    const int tx = tid & 15, ty = tid >> 4;
    for (int t = 0; t < rtiles * ctiles; ++t) {
      const int r0 = (t / ctiles) * TR, q0 = c0 + (t % ctiles) * 64;  // r0 counts from row c0
      for (int q = tid; q < NB * 64; q += NT) {
        const int l = q / 64, cc = q % 64;
        Bs[l][cc] = (q0 + cc < N && l < kb) ? A[(long long)(k0 + l) * N + q0 + cc] : (T)0;
      }
      __syncthreads();
      T acc[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = (T)0;
      if (r0 + ty * 4 < mt) {
        const T* Lp = P + (kb + r0 + ty * 4) * LD;
#pragma unroll 4
        for (int l = 0; l < kb; ++l) {
          T a[4], bb[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = (r0 + ty * 4 + i < mt) ? Lp[i * LD + l] : (T)0;
#pragma unroll
          for (int j = 0; j < 4; ++j) bb[j] = Bs[l][tx * 4 + j];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * bb[j];
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = c0 + r0 + ty * 4 + i;
        if (r >= N) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int cc = q0 + tx * 4 + j;
          if (cc < N) A[(long long)r * N + cc] -= acc[i][j];
        }
      }
      __syncthreads();
    }
  }
}

// x <- (LU)^-1 P x in place (x in shared memory, FP64 arithmetic): the row
// swaps, then unit-lower and upper block substitution (32-row diagonal blocks
// by warp 0 with shuffles, the rest by all threads).
template <class T>
__device__ void cta_lu_solve(const T* LU, int N, const int* piv, double* x) {
  if (threadIdx.x == 0)
    for (int k = 0; k < N; ++k) {
      const int p = piv[k];
      if (p != k) {
        const double t = x[k];
        x[k] = x[p];
        x[p] = t;
      }
    }
  __syncthreads();
  // Full 32-column blocks take unrolled loops (the same operations in the
  // same order): the loads of a row segment, which do not depend on the
  // substitution chain, then issue together instead of a few at a time.
  for (int J0 = 0; J0 < N; J0 += 32) {
    const int nb = min(32, N - J0);
    if (threadIdx.x < 32) {
      const int q = threadIdx.x;
      double v = q < nb ? x[J0 + q] : 0.0;
      if (nb == 32) {
        const T* a = LU + (long long)(J0 + q) * N + J0;
#pragma unroll
        for (int l = 0; l < 32; ++l) {
          const double xl = __shfl_sync(0xffffffffu, v, l);
          if (q > l) v -= (double)a[l] * xl;
        }
      } else {
        for (int l = 0; l < nb; ++l) {
          const double xl = __shfl_sync(0xffffffffu, v, l);
          if (q > l && q < nb) v -= (double)LU[(long long)(J0 + q) * N + J0 + l] * xl;
        }
      }
      if (q < nb) x[J0 + q] = v;
    }
    __syncthreads();
    if (nb == 32) {
#pragma unroll 2
      for (int i = J0 + 32 + threadIdx.x; i < N; i += blockDim.x) {
        const T* a = LU + (long long)i * N + J0;
        double s = x[i];
#pragma unroll
        for (int l = 0; l < 32; ++l) s -= (double)a[l] * x[J0 + l];
        x[i] = s;
      }
    } else {
      for (int i = J0 + nb + threadIdx.x; i < N; i += blockDim.x) {
        double s = x[i];
        for (int l = 0; l < nb; ++l) s -= (double)LU[(long long)i * N + J0 + l] * x[J0 + l];
        x[i] = s;
      }
    }
    __syncthreads();
  }
  for (int J1 = N; J1 > 0; J1 -= 32) {
    const int J0 = max(0, J1 - 32), nb = J1 - J0;
    if (threadIdx.x < 32) {
      const int q = threadIdx.x;
      double v = q < nb ? x[J0 + q] : 0.0;
      if (nb == 32) {
        const T* a = LU + (long long)(J0 + q) * N + J0;
#pragma unroll
        for (int l = 31; l >= 0; --l) {
          if (q == l) v /= (double)a[l];
          const double xl = __shfl_sync(0xffffffffu, v, l);
          if (q < l) v -= (double)a[l] * xl;
        }
      } else {
        for (int l = nb - 1; l >= 0; --l) {
          if (q == l) v /= (double)LU[(long long)(J0 + l) * N + J0 + l];
          const double xl = __shfl_sync(0xffffffffu, v, l);
          if (q < l) v -= (double)LU[(long long)(J0 + q) * N + J0 + l] * xl;
        }
      }
      if (q < nb) x[J0 + q] = v;
    }
    __syncthreads();
    if (nb == 32) {
#pragma unroll 2
      for (int i = threadIdx.x; i < J0; i += blockDim.x) {
        const T* a = LU + (long long)i * N + J0;
        double s = x[i];
#pragma unroll
        for (int l = 0; l < 32; ++l) s -= (double)a[l] * x[J0 + l];
        x[i] = s;
      }
    } else {
      for (int i = threadIdx.x; i < J0; i += blockDim.x) {
        double s = x[i];
        for (int l = 0; l < nb; ++l) s -= (double)LU[(long long)i * N + J0 + l] * x[J0 + l];
        x[i] = s;
      }
    }
    __syncthreads();
  }
}

template <int NT>
__device__ double cta_sum(double v) {
  __shared__ double sh[NT / 32];
  for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0;
  for (int w = 0; w < NT / 32; ++w) t += sh[w];
  return t;
}

// Refinement sweeps a stale factorisation may spend before the case is
// factored again, and the contraction each sweep must reach.
constexpr int kStaleSweeps = 12;
constexpr double kStaleContraction = 0.5;

// One CTA per case: G = A^-1 b.  FP64 form: LU of A in place.  Mixed form:
// sweeps g += (LU)^-1 (b - A g) with the FP64 residual until
// ||b - A g|| <= tol ||b||, where LU are FP32 factors of A.  With stale
// factors allowed, a case that already holds factors (of an earlier step's
// matrix) first refines from its previous circulation with them; only when
// that does not reach the tolerance, or a sweep contracts the residual by less
// than kStaleContraction, is the FP32 copy of the current A factored again
// (each case decides for itself; refac counts the factorisations).
template <class T>
__global__ void __launch_bounds__(SolveCfg<T>::kThreads) b_solve_kernel(const BCase* __restrict__ cs, double* A64, float* F32,
                                                                int* piv_all, const double* rhs, double* gamma,
                                                                const double* gamma_hist, const long long* d_step,
                                                                int max_sweeps, double tol, int stale,
                                                                int* has_factor, unsigned long long* refac,
                                                                int* sweeps_out, double* res_out, int* status,
                                                                const int* __restrict__ order) {
  constexpr int NT = SolveCfg<T>::kThreads;
  extern __shared__ double sm[];
  // CTA i takes the i-th largest case: with more cases than SMs the largest
  // start first instead of forming the launch's last wave
  const int ci = order[blockIdx.x];
  const BCase& b = cs[ci];
  const int N = b.N;
  double* x = sm;
  double* r = sm + N;
  T* panel = reinterpret_cast<T*>(sm + 2 * N);
  double* A = A64 + b.mat_off;
  int* piv = piv_all + b.ring_off;
  const double* bb = rhs + b.ring_off;
  int sweeps = 0;
  double rel = 0;
  if constexpr (sizeof(T) == 4) {
    T* LU = F32 + b.mat_off;
    double bn = 0;
    for (int i = threadIdx.x; i < N; i += NT) bn += bb[i] * bb[i];
    bn = sqrt(cta_sum<NT>(bn));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // r = b - A x (FP64), returns ||r|| / ||b|| (same value in every thread)
    auto residual = [&]() -> double {
      // four rows per warp at a time, so that enough loads of A are in
      // flight for one SM to stream the matrix
      constexpr int kW = NT / 32;
      for (int i0 = wid; i0 < N; i0 += 4 * kW) {
        const double* a0 = A + (long long)i0 * N;
        const bool v1 = i0 + kW < N, v2 = i0 + 2 * kW < N, v3 = i0 + 3 * kW < N;
        const double* a1 = v1 ? a0 + (long long)kW * N : a0;
        const double* a2 = v2 ? a0 + 2LL * kW * N : a0;
        const double* a3 = v3 ? a0 + 3LL * kW * N : a0;
        double c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll 8
        for (int j = lane; j < N; j += 32) {
          const double xj = x[j];
          c0 += a0[j] * xj;
          c1 += a1[j] * xj;
          c2 += a2[j] * xj;
          c3 += a3[j] * xj;
        }
        for (int off = 16; off; off >>= 1) {
          c0 += __shfl_down_sync(0xffffffffu, c0, off);
          c1 += __shfl_down_sync(0xffffffffu, c1, off);
          c2 += __shfl_down_sync(0xffffffffu, c2, off);
          c3 += __shfl_down_sync(0xffffffffu, c3, off);
        }
        if (lane == 0) {
          r[i0] = bb[i0] - c0;
          if (v1) r[i0 + kW] = bb[i0 + kW] - c1;
          if (v2) r[i0 + 2 * kW] = bb[i0 + 2 * kW] - c2;
          if (v3) r[i0 + 3 * kW] = bb[i0 + 3 * kW] - c3;
        }
      }
      __syncthreads();
      double rn = 0;
      for (int i = threadIdx.x; i < N; i += NT) rn += r[i] * r[i];
      rn = sqrt(cta_sum<NT>(rn));
      return bn > 0 ? rn / bn : 0.0;
    };
    auto sweep = [&]() {
      cta_lu_solve<T>(LU, N, piv, r);
      for (int i = threadIdx.x; i < N; i += NT) x[i] += r[i];
      __syncthreads();
    };
    bool done = false;
    if (stale && has_factor[ci]) {
      // refine from the extrapolation 2 G(s-1) - G(s-2) (from G(s-1) before step 2)
      const bool extrap = *d_step >= 2;
      for (int i = threadIdx.x; i < N; i += NT)
        x[i] = extrap ? 2.0 * gamma[b.ring_off + i] - gamma_hist[b.ring_off + i] : gamma[b.ring_off + i];
      __syncthreads();
      rel = residual();
      double prev = rel;
      for (int k = 0; k < kStaleSweeps && rel > tol && rel == rel; ++k) {
        sweep();
        ++sweeps;
        rel = residual();
        if (!(rel < kStaleContraction * prev)) break;
        prev = rel;
      }
      done = rel <= tol;
    }
    if (!done) {
      for (long long q = threadIdx.x; q < (long long)N * N; q += NT) LU[q] = (float)A[q];
      __syncthreads();
      cta_lu_panel_smem<T>(LU, N, piv, status, panel);
      if (threadIdx.x == 0) {
        has_factor[ci] = 1;
        atomicAdd(refac, 1ull);
      }
      for (int i = threadIdx.x; i < N; i += NT) x[i] = bb[i];
      __syncthreads();
      cta_lu_solve<T>(LU, N, piv, x);
      sweeps = 0;
      while (true) {
        rel = residual();
        if (rel <= tol || sweeps >= max_sweeps || !(rel == rel)) break;
        sweep();
        ++sweeps;
      }
    }
    if (threadIdx.x == 0 && !(rel <= tol)) status[3] = 1;
  } else {
    cta_lu_panel_smem<T>(A, N, piv, status, panel);
    if (threadIdx.x == 0) atomicAdd(refac, 1ull);
    for (int i = threadIdx.x; i < N; i += NT) x[i] = bb[i];
    __syncthreads();
    cta_lu_solve<T>(A, N, piv, x);
  }
  bool finite = true;
  for (int i = threadIdx.x; i < N; i += NT) {
    gamma[b.ring_off + i] = x[i];
    if (!isfinite(x[i])) finite = false;
  }
  if (!finite) status[2] = 1;
  if (threadIdx.x == 0) {
    sweeps_out[ci] = sweeps;
    res_out[ci] = rel;
  }
}

// ------------------------------------------------------------------- loads
__global__ void b_line_prep_kernel(const BCase* __restrict__ cs, BPrefix P, int n, const long long* d_step,
                                   const double* pos, const double* pos_init, double* lx, double* ly, double* lz,
                                   double* line_uls) {
  const long long s = *d_step;
  const long long total = P.line[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const BCase& b = cs[find_case(P.line, n, g)];
    const WingShape ws = shape_of(b);
    long long a, e;
    line_nodes(ws, 0, (int)(g - b.line_off), a, e);
    const double* ps = pos + 3 * b.node_off;
    const double* p0 = pos_init + 3 * b.node_off;
    const d3 mp = dvs(add(ld3(ps + 3 * a), ld3(ps + 3 * e)), 2);
    const d3 mp0 = dvs(add(ld3(p0 + 3 * a), ld3(p0 + 3 * e)), 2);
    lx[g] = mp.x;
    ly[g] = mp.y;
    lz[g] = mp.z;
    st3(line_uls + 3 * g, morph_velocity(b.kin, mp0, (double)s * b.dt));
  }
}

constexpr int kLoadThreads = 256;

__device__ double load_sum(double v, double* sh) {
  for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0;
  for (int w = 0; w < kLoadThreads / 32; ++w) t += sh[w];
  return t;
}

// CalcLoad (simple_simulator.cpp:195-233) per case: JoukowskiSteady over the
// lines plus JoukowskiUnsteady, C = F / (0.5 |ff|^2 chord span); row
// (t, CD = C.x, CL = C.z) of this step.
__global__ void __launch_bounds__(kLoadThreads) b_loads_kernel(const BCase* __restrict__ cs, int n,
                                                               const long long* d_step, const double* pos,
                                                               const double* gamma, const double* gamma_prev,
                                                               const double* normal, const double* area,
                                                               const double* vx, const double* vy, const double* vz,
                                                               const double* line_uls, double* loads) {
  __shared__ double sh[kLoadThreads / 32];
  const long long s = *d_step;
  const int c = blockIdx.x;
  const BCase& b = cs[c];
  const WingShape ws = shape_of(b);
  const double* ps = pos + 3 * b.node_off;
  const double* gm = gamma + b.ring_off;
  const d3 mff = mk(-b.ff[0], -b.ff[1], -b.ff[2]);
  double f[3] = {0, 0, 0};
  for (int q = threadIdx.x; q < b.lines; q += kLoadThreads) {
    const long long k = b.line_off + q;
    long long a, e;
    line_nodes(ws, 0, q, a, e);
    const d3 dl = sub(ld3(ps + 3 * e), ld3(ps + 3 * a));
    const d3 U = sub(add(mff, mk(vx[k], vy[k], vz[k])), ld3(line_uls + 3 * k));
    const d3 df = scl(cross(U, dl), line_strength(ws, gm, 0, q));
    f[0] += df.x;
    f[1] += df.y;
    f[2] += df.z;
  }
  const double dt = b.dt;
  for (int p = threadIdx.x; p < b.N; p += kLoadThreads) {
    const long long K = b.ring_off + p;
    const double dgdt = (gamma[K] - gamma_prev[K]) / dt;
    const d3 df = scl(scl(ld3(normal + 3 * K), dgdt), area[K]);
    f[0] += df.x;
    f[1] += df.y;
    f[2] += df.z;
  }
  const double Fx = load_sum(f[0], sh);
  const double Fz = load_sum(f[2], sh);
  if (threadIdx.x == 0) {
    const double Q = norm(mff);
    const double den = 0.5 * Q * Q * b.area_ref;
    double* row = loads + (s * n + c) * 3;
    row[0] = (double)s * dt;
    row[1] = Fx / den;
    row[2] = Fz / den;
  }
}

// ----------------------------------------------------------------- advect
__global__ void b_gather_wake_kernel(const BCase* __restrict__ cs, BPrefix P, int n, int cap,
                                     const long long* d_step, const double* wpos, double* tx, double* ty,
                                     double* tz) {
  const long long s = *d_step;
  const long long start = cap - 1 - s;
  const long long total = P.wtgt[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const BCase& b = cs[find_case(P.wtgt, n, g)];
    const long long k = g - b.wtgt_off;
    const long long i = k / (b.C + 1) + 1;
    if (i > s) continue;
    const int j = (int)(k % (b.C + 1));
    const double* p = wpos + 3 * (b.wnode_off + (start + i) * (b.C + 1) + j);
    tx[g] = p[0];
    ty[g] = p[1];
    tz[g] = p[2];
  }
}

// u = -ff + U (rows >= 1) or -ff (row 0, src/advect.h:41-45); Euler
// (src/advect.cpp:11-22) or the two RK2 stages (:24-80).
__global__ void b_advect_kernel(const BCase* __restrict__ cs, BPrefix P, int n, int cap, const long long* d_step,
                                int mode, int ignore, double* x, double* pos2, double* k1, const double* vx,
                                const double* vy, const double* vz) {
  const long long s = *d_step;
  const long long start = cap - 1 - s;
  const long long total = P.wnode[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int c = find_case(P.wnode, n, g);
    const BCase& b = cs[c];
    const long long k = g - P.wnode[c];
    const long long i = k / (b.C + 1);
    if (i > s) continue;
    const int j = (int)(k % (b.C + 1));
    const long long Pn = 3 * (b.wnode_off + (start + i) * (b.C + 1) + j);
    const d3 mff = mk(-b.ff[0], -b.ff[1], -b.ff[2]);
    d3 u = mff;
    if (i >= 1) {
      const long long ti = b.wtgt_off + (i - 1) * (b.C + 1) + j;
      u = add(mff, mk(vx[ti], vy[ti], vz[ti]));
    }
    const d3 xp = ld3(x + Pn);
    const double dt = b.dt;
    if (mode == kAdvEuler) {
      st3(x + Pn, add(xp, scl(u, dt)));
    } else if (mode == kAdvRK2K1) {
      st3(k1 + Pn, u);
      st3(pos2 + Pn, add(xp, scl(u, dt)));
    } else {
      const d3 a = ld3(k1 + Pn);
      st3(x + Pn, i > ignore ? add(xp, dvs(scl(add(a, u), dt), 2)) : add(xp, scl(a, dt)));
    }
  }
}

// Synthetic wake of the tile autotuner: every case's trailing edge convected
// by its forward flight for s steps with a gentle vertical wave (node rows
// 0..s of the layout above), the shape of a late step's wake.
__global__ void b_synth_wake_kernel(const BCase* __restrict__ cs, BPrefix P, int n, int cap, long long s,
                                    const double* pos_init, double* wpos) {
  const long long total = P.wnode[n];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const BCase& b = cs[find_case(P.wnode, n, g)];
    const long long local = g - b.wnode_off;
    const long long i = local / (b.C + 1) - (cap - 1 - s);
    if (i < 0) continue;
    const int j = (int)(local % (b.C + 1));
    const d3 te = ld3(pos_init + 3 * (b.node_off + (long long)b.R * (b.C + 1) + j));
    const double t = (double)i * b.dt;
    st3(wpos + 3 * g, add(te, mk(-b.ff[0] * t, -b.ff[1] * t, -b.ff[2] * t + 0.05 * sin(0.3 * (double)i))));
  }
}

__global__ void b_step_end_kernel(long long* d_step) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *d_step += 1;
}

}  // namespace
}  // namespace uvlm

using namespace uvlm;

struct uvlm_batch {
  uvlm_batch_config cfg{};
  std::string err;
  int n = 0, cap = 0, num_sms = 148, grid = 0;
  NBodyBatchGrids nb_grids;
  int64_t steps_done = 0;
  std::vector<BCase> hc;
  std::vector<long long> pre[7];
  long long tot_nodes = 0, tot_rings = 0, tot_lines = 0, tot_te = 0, tot_rec = 0, tot_wnode = 0, tot_wtgt = 0,
            tot_mat = 0;
  int max_N = 0;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t launches_per_step = 0;
  // device
  BCase* d_cases = nullptr;
  long long* d_pre = nullptr;  // 7 prefix arrays of n + 1
  long long* d_step = nullptr;
  double *d_pos_init = nullptr, *d_pos = nullptr, *d_gamma = nullptr, *d_gamma_prev = nullptr;
  double* d_gamma_hist = nullptr;
  double *d_cx = nullptr, *d_cy = nullptr, *d_cz = nullptr, *d_normal = nullptr, *d_area = nullptr,
         *d_uls = nullptr, *d_rhs = nullptr;
  double *d_lx = nullptr, *d_ly = nullptr, *d_lz = nullptr, *d_line_uls = nullptr;
  double *d_wpos = nullptr, *d_wpos2 = nullptr, *d_k1 = nullptr, *d_wgamma = nullptr;
  double *d_wtx = nullptr, *d_wty = nullptr, *d_wtz = nullptr;
  double *d_vx = nullptr, *d_vy = nullptr, *d_vz = nullptr;
  double* d_A64 = nullptr;
  float* d_F32 = nullptr;
  int* d_piv = nullptr;
  AsmTile* d_tiles = nullptr;
  int n_tiles = 0;
  void* d_rec = nullptr;
  double* d_partial = nullptr;
  long long partial_cap = 0;
  NBodyBatchInput* d_in = nullptr;
  NBodyBatchPlan* d_plan = nullptr;
  long long* d_totals = nullptr;
  int* d_status = nullptr;
  int* d_sweeps = nullptr;
  int* d_solve_order = nullptr;          // cases by decreasing N (the solve's CTA order)
  int* d_has_factor = nullptr;           // per case: FP32 factors held (stale reuse)
  unsigned long long* d_refac = nullptr;  // factorisations so far
  double* d_res = nullptr;
  double* d_loads = nullptr;

  bool mixed() const { return cfg.precision == UVLM_PRECISION_MIXED; }
  NBodyPrec prec() const { return mixed() ? kNBodyFP32 : kNBodyFP64; }
  BPrefix prefixes() const {
    const long long* p = d_pre;
    const long long m = n + 1;
    return BPrefix{p, p + m, p + 2 * m, p + 3 * m, p + 4 * m, p + 5 * m, p + 6 * m};
  }
  int fail_with(const Error& e) {
    if (e.code) err = e.msg;
    return e.code;
  }
  Error alloc(const uvlm_batch_case* cases);
  Error build_records(int with_bound, const double* wsrc);
  Error tune_tiles();
  Error enqueue_step();
  Error nbody(int stage, const double* tx, const double* ty, const double* tz);
  void release();
};

namespace {
template <class T>
Error balloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  UVLM_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count));
  return ok();
}
}  // namespace

Error uvlm_batch::alloc(const uvlm_batch_case* cases) {
  cap = (int)cfg.max_steps + 1;
  for (auto& v : pre) v.assign(n + 1, 0);
  hc.resize(n);
  std::vector<double> nodes;
  std::vector<AsmTile> tiles;
  long long off[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int c = 0; c < n; ++c) {
    const uvlm_batch_case& u = cases[c];
    BCase& b = hc[c];
    b.R = (int)u.rows;
    b.C = (int)u.cols;
    b.N = b.R * b.C;
    b.lines = b.R * (2 * b.C + 1);
    const long long nn = (long long)(b.R + 1) * (b.C + 1);
    b.node_off = off[0];
    b.ring_off = off[1];
    b.line_off = off[2];
    b.rec_off = off[4];
    b.wnode_off = off[5];
    b.wring_off = off[7];
    b.wtgt_off = off[6];
    b.mat_off = tot_mat;
    for (int d = 0; d < 3; ++d) b.ff[d] = u.forward_flight[d];
    b.dt = u.dt;
    b.area_ref = u.chord * u.span;
    b.kin = u.kin;
    for (int d = 0; d < 3; ++d) b.kin.origin[d] = u.origin[d];
    const long long cnt[7] = {nn, b.N, b.lines, b.C + 1, nn + (long long)cap * (b.C + 1), (long long)cap * (b.C + 1),
                              (long long)(cap - 1) * (b.C + 1)};
    for (int k = 0; k < 7; ++k) {
      pre[k][c] = off[k];
      off[k] += cnt[k];
    }
    off[7] += (long long)cap * b.C;
    tot_mat += (long long)b.N * b.N;
    max_N = std::max(max_N, b.N);
    uvlm_wing_desc w{};
    w.chord = u.chord;
    w.span = u.span;
    w.rows = u.rows;
    w.cols = u.cols;
    for (int d = 0; d < 3; ++d) w.origin[d] = u.origin[d];
    w.chebyshev_chord = u.chebyshev_chord;
    w.chebyshev_span = u.chebyshev_span;
    auto v = whole_wing_nodes(w);
    nodes.insert(nodes.end(), v.begin(), v.end());
    // assembly tiles: runs of (collocation point, node column) positions
    const long long positions = (long long)b.N * (b.C + 1);
    for (long long p0 = 0; p0 < positions; p0 += kBAsmTilePositions)
      tiles.push_back(AsmTile{c, p0, std::min(positions, p0 + kBAsmTilePositions)});
  }
  for (int k = 0; k < 7; ++k) pre[k][n] = off[k];
  tot_nodes = off[0];
  tot_rings = off[1];
  tot_lines = off[2];
  tot_te = off[3];
  tot_rec = off[4];
  tot_wnode = off[5];
  tot_wtgt = off[6];
  const long long tot_wring = off[7];
  n_tiles = (int)tiles.size();

  UVLM_TRY(balloc(&d_cases, n));
  UVLM_TRY(balloc(&d_pre, 7 * (size_t)(n + 1)));
  UVLM_TRY(balloc(&d_step, 1));
  UVLM_TRY(balloc(&d_pos_init, 3 * tot_nodes));
  UVLM_TRY(balloc(&d_pos, 3 * tot_nodes));
  UVLM_TRY(balloc(&d_gamma, tot_rings));
  UVLM_TRY(balloc(&d_gamma_prev, tot_rings));
  UVLM_TRY(balloc(&d_gamma_hist, tot_rings));
  UVLM_TRY(balloc(&d_cx, tot_rings));
  UVLM_TRY(balloc(&d_cy, tot_rings));
  UVLM_TRY(balloc(&d_cz, tot_rings));
  UVLM_TRY(balloc(&d_normal, 3 * tot_rings));
  UVLM_TRY(balloc(&d_area, tot_rings));
  UVLM_TRY(balloc(&d_uls, 3 * tot_rings));
  UVLM_TRY(balloc(&d_rhs, tot_rings));
  UVLM_TRY(balloc(&d_lx, tot_lines));
  UVLM_TRY(balloc(&d_ly, tot_lines));
  UVLM_TRY(balloc(&d_lz, tot_lines));
  UVLM_TRY(balloc(&d_line_uls, 3 * tot_lines));
  UVLM_TRY(balloc(&d_wpos, 3 * tot_wnode));
  UVLM_TRY(balloc(&d_wgamma, tot_wring));
  if (cfg.advection == UVLM_ADVECT_RK2) {
    UVLM_TRY(balloc(&d_wpos2, 3 * tot_wnode));
    UVLM_TRY(balloc(&d_k1, 3 * tot_wnode));
  }
  UVLM_TRY(balloc(&d_wtx, tot_wtgt));
  UVLM_TRY(balloc(&d_wty, tot_wtgt));
  UVLM_TRY(balloc(&d_wtz, tot_wtgt));
  const long long nv = std::max({tot_rings, tot_lines, tot_wtgt});
  UVLM_TRY(balloc(&d_vx, nv));
  UVLM_TRY(balloc(&d_vy, nv));
  UVLM_TRY(balloc(&d_vz, nv));
  UVLM_TRY(balloc(&d_A64, tot_mat));
  if (mixed()) UVLM_TRY(balloc(&d_F32, tot_mat));
  UVLM_TRY(balloc(&d_piv, tot_rings));
  UVLM_TRY(balloc(&d_tiles, n_tiles));
  UVLM_CUDA_TRY(cudaMalloc(&d_rec, (size_t)tot_rec * (mixed() ? sizeof(RecF) : sizeof(RecD))));
  // partial sums: the largest stage at the last step bounds every step
  {
    const long long s = cfg.max_steps - 1;
    std::vector<NBodyBatchInput> in(n);
    for (int stage = 0; stage < 3; ++stage) {
      for (int c = 0; c < n; ++c) {
        const BCase& b = hc[c];
        NBodyBatchInput x{};
        const long long nb = (long long)(b.R + 1) * (b.C + 1);
        const SourceBlock wake{b.rec_off + nb, 1, (int)(s + 1), b.C};
        if (stage == kStageRhs) {
          x.blocks[0] = wake;
          x.n_blocks = 1;
          x.n_tgt = b.N;
        } else {
          x.blocks[0] = SourceBlock{b.rec_off, 1, b.R + 1, b.C};
          x.blocks[1] = wake;
          x.n_blocks = 2;
          x.n_tgt = stage == kStageLoads ? b.lines : s * (b.C + 1);
        }
        in[c] = x;
      }
      partial_cap = std::max(partial_cap, nbody_batch_partial_doubles(prec(), in.data(), n));
    }
  }
  UVLM_TRY(balloc(&d_partial, partial_cap));
  UVLM_TRY(balloc(&d_in, n));
  UVLM_TRY(balloc(&d_plan, n));
  UVLM_TRY(balloc(&d_totals, 4));
  UVLM_TRY(balloc(&d_status, 4));
  UVLM_TRY(balloc(&d_sweeps, n));
  UVLM_TRY(balloc(&d_solve_order, n));
  UVLM_TRY(balloc(&d_has_factor, n));
  UVLM_TRY(balloc(&d_refac, 1));
  UVLM_TRY(balloc(&d_res, n));
  UVLM_TRY(balloc(&d_loads, (size_t)cfg.max_steps * n * 3));

  std::vector<long long> flat;
  for (int k = 0; k < 7; ++k) flat.insert(flat.end(), pre[k].begin(), pre[k].end());
  UVLM_CUDA_TRY(cudaMemcpy(d_cases, hc.data(), sizeof(BCase) * n, cudaMemcpyHostToDevice));
  {
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return hc[a].N > hc[b].N; });
    UVLM_CUDA_TRY(cudaMemcpy(d_solve_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  }
  UVLM_CUDA_TRY(cudaMemcpy(d_pre, flat.data(), sizeof(long long) * flat.size(), cudaMemcpyHostToDevice));
  UVLM_CUDA_TRY(cudaMemcpy(d_tiles, tiles.data(), sizeof(AsmTile) * tiles.size(), cudaMemcpyHostToDevice));
  UVLM_CUDA_TRY(cudaMemcpy(d_pos_init, nodes.data(), sizeof(double) * nodes.size(), cudaMemcpyHostToDevice));
  UVLM_CUDA_TRY(cudaMemcpy(d_pos, nodes.data(), sizeof(double) * nodes.size(), cudaMemcpyHostToDevice));
  UVLM_CUDA_TRY(cudaMemset(d_step, 0, sizeof(long long)));
  UVLM_CUDA_TRY(cudaMemset(d_gamma, 0, sizeof(double) * tot_rings));
  UVLM_CUDA_TRY(cudaMemset(d_gamma_prev, 0, sizeof(double) * tot_rings));
  UVLM_CUDA_TRY(cudaMemset(d_gamma_hist, 0, sizeof(double) * tot_rings));
  UVLM_CUDA_TRY(cudaMemset(d_wpos, 0, sizeof(double) * 3 * tot_wnode));
  UVLM_CUDA_TRY(cudaMemset(d_wgamma, 0, sizeof(double) * tot_wring));
  UVLM_CUDA_TRY(cudaMemset(d_status, 0, sizeof(int) * 4));
  UVLM_CUDA_TRY(cudaMemset(d_has_factor, 0, sizeof(int) * n));
  UVLM_CUDA_TRY(cudaMemset(d_refac, 0, sizeof(unsigned long long)));
  UVLM_CUDA_TRY(cudaMemset(d_loads, 0, sizeof(double) * (size_t)cfg.max_steps * n * 3));
  const size_t solve_smem = sizeof(double) * 2 * (size_t)max_N + panel_smem_bytes(max_N, mixed() ? 4 : 8);
  if (mixed())
    UVLM_CUDA_TRY(cudaFuncSetAttribute(b_solve_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)solve_smem));
  else
    UVLM_CUDA_TRY(cudaFuncSetAttribute(b_solve_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)solve_smem));
  nb_grids = nbody_batch_grids(prec(), num_sms);
  grid = num_sms * 8;
  return ok();
}

Error uvlm_batch::nbody(int stage, const double* tx, const double* ty, const double* tz) {
  b_nbody_inputs_kernel<<<(n + 127) / 128, 128, 0, st>>>(d_cases, n, d_step, stage, d_in);
  UVLM_LAUNCH_CHECK();
  return nbody_batch_eval(prec(), d_in, n, tx, ty, tz, d_vx, d_vy, d_vz, d_rec, d_partial, partial_cap, d_plan,
                          d_totals, d_status, nb_grids, st);
}

Error uvlm_batch::build_records(int with_bound, const double* wsrc) {
  const BPrefix P = prefixes();
  if (mixed())
    b_records_kernel<RecF><<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, with_bound, d_pos, d_gamma, wsrc,
                                                d_wgamma, reinterpret_cast<RecF*>(d_rec));
  else
    b_records_kernel<RecD><<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, with_bound, d_pos, d_gamma, wsrc,
                                                d_wgamma, reinterpret_cast<RecD*>(d_rec));
  UVLM_LAUNCH_CHECK();
  return ok();
}

// Tile autotuner of the batched N-body (before the first step, outside any
// graph capture): the advection stage of the last step the batch can run,
// on a synthetic wake of that length (b_synth_wake_kernel), is timed with
// every compiled FP32 tile; the fastest is kept (the default unless another
// is more than 3% faster) and every later step, captured once as a graph,
// runs it.  The wake buffers and the step counter are cleared afterwards.
Error uvlm_batch::tune_tiles() {
  if (!mixed()) return ok();
  if (cfg.nbody_tile >= 0) {
    nb_grids.tile = cfg.nbody_tile;
    return ok();
  }
  const long long s = cfg.max_steps - 1;
  if (s < 2) return ok();
  const BPrefix P = prefixes();
  b_synth_wake_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, s, d_pos_init, d_wpos);
  UVLM_LAUNCH_CHECK();
  UVLM_CUDA_TRY(cudaMemcpyAsync(d_step, &s, sizeof(s), cudaMemcpyHostToDevice, st));
  UVLM_TRY(build_records(1, d_wpos));
  b_gather_wake_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, d_wpos, d_wtx, d_wty, d_wtz);
  UVLM_LAUNCH_CHECK();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  UVLM_CUDA_TRY(cudaEventCreate(&e0));
  UVLM_CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f;
  int chosen = 0;
  Error err = ok();
  for (int t = 0; t < kNumBatchTilesF && !err.code; ++t) {
    nb_grids.tile = t;
    float ms = 0;
    for (int rep = 0; rep < 3 && !err.code; ++rep) {  // the first run warms caches and module state
      cudaEventRecord(e0, st);
      err = nbody(kStageAdvect, d_wtx, d_wty, d_wtz);
      cudaEventRecord(e1, st);
      if (!err.code && cudaEventSynchronize(e1) != cudaSuccess) err = fail(kErrCuda, "tile autotune");
      if (!err.code) cudaEventElapsedTime(&ms, e0, e1);
    }
    const float score = t == 0 ? ms / 1.03f : ms;
    if (!err.code && score < best) {
      best = score;
      chosen = t;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  nb_grids.tile = chosen;
  UVLM_TRY(err);
  const long long zero = 0;
  UVLM_CUDA_TRY(cudaMemsetAsync(d_wpos, 0, sizeof(double) * 3 * (size_t)tot_wnode, st));
  UVLM_CUDA_TRY(cudaMemcpyAsync(d_step, &zero, sizeof(zero), cudaMemcpyHostToDevice, st));
  UVLM_CUDA_TRY(cudaStreamSynchronize(st));
  return ok();
}

Error uvlm_batch::enqueue_step() {
  const BPrefix P = prefixes();
  auto records = [&](int with_bound, const double* wsrc) -> Error { return build_records(with_bound, wsrc); };
  b_begin_kernel<<<grid, 256, 0, st>>>(P.ring, n, d_gamma, d_gamma_prev, d_gamma_hist);
  UVLM_LAUNCH_CHECK();
  b_kinematics_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, d_step, d_pos_init, d_pos);
  UVLM_LAUNCH_CHECK();
  b_shed_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, d_pos, d_gamma, d_wpos, d_wgamma);
  UVLM_LAUNCH_CHECK();
  b_geometry_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, d_step, d_pos, d_pos_init, d_cx, d_cy, d_cz, d_normal,
                                          d_area, d_uls);
  UVLM_LAUNCH_CHECK();
  b_assemble_kernel<<<n_tiles, kBAsmThreads, 0, st>>>(d_cases, d_tiles, d_pos, d_cx, d_cy, d_cz, d_normal, d_A64);
  UVLM_LAUNCH_CHECK();
  // RHS: wake normal wash at the collocation points
  UVLM_TRY(records(0, d_wpos));
  UVLM_TRY(nbody(kStageRhs, d_cx, d_cy, d_cz));
  b_rhs_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, d_vx, d_vy, d_vz, d_uls, d_normal, d_rhs);
  UVLM_LAUNCH_CHECK();
  // solve
  const size_t smem = sizeof(double) * 2 * (size_t)max_N + panel_smem_bytes(max_N, mixed() ? 4 : 8);
  if (mixed())
    b_solve_kernel<float><<<n, SolveCfg<float>::kThreads, smem, st>>>(d_cases, d_A64, d_F32, d_piv, d_rhs, d_gamma,
                                                          d_gamma_hist, d_step, cfg.refine_max_iter, cfg.refine_tol, cfg.stale_factors,
                                                          d_has_factor, d_refac, d_sweeps, d_res, d_status, d_solve_order);
  else
    b_solve_kernel<double><<<n, SolveCfg<double>::kThreads, smem, st>>>(d_cases, d_A64, d_F32, d_piv, d_rhs, d_gamma,
                                                           d_gamma_hist, d_step, 0, 0.0,
                                                           0, d_has_factor, d_refac, d_sweeps, d_res, d_status, d_solve_order);
  UVLM_LAUNCH_CHECK();
  // loads: line velocities from the bound sheet (new circulation) and the wake
  b_line_prep_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, d_step, d_pos, d_pos_init, d_lx, d_ly, d_lz, d_line_uls);
  UVLM_LAUNCH_CHECK();
  UVLM_TRY(records(1, d_wpos));
  UVLM_TRY(nbody(kStageLoads, d_lx, d_ly, d_lz));
  b_loads_kernel<<<n, kLoadThreads, 0, st>>>(d_cases, n, d_step, d_pos, d_gamma, d_gamma_prev, d_normal, d_area,
                                             d_vx, d_vy, d_vz, d_line_uls, d_loads);
  UVLM_LAUNCH_CHECK();
  // advection: the same sources as the loads
  b_gather_wake_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, d_wpos, d_wtx, d_wty, d_wtz);
  UVLM_LAUNCH_CHECK();
  UVLM_TRY(nbody(kStageAdvect, d_wtx, d_wty, d_wtz));
  if (cfg.advection == UVLM_ADVECT_RK2) {
    b_advect_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, kAdvRK2K1, cfg.rk_ignore_rows, d_wpos, d_wpos2,
                                          d_k1, d_vx, d_vy, d_vz);
    UVLM_LAUNCH_CHECK();
    UVLM_TRY(records(0, d_wpos2));
    b_gather_wake_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, d_wpos2, d_wtx, d_wty, d_wtz);
    UVLM_LAUNCH_CHECK();
    UVLM_TRY(nbody(kStageAdvect, d_wtx, d_wty, d_wtz));
    b_advect_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, kAdvRK2Upd, cfg.rk_ignore_rows, d_wpos, d_wpos2,
                                          d_k1, d_vx, d_vy, d_vz);
  } else {
    b_advect_kernel<<<grid, 256, 0, st>>>(d_cases, P, n, cap, d_step, kAdvEuler, cfg.rk_ignore_rows, d_wpos, d_wpos2,
                                          d_k1, d_vx, d_vy, d_vz);
  }
  UVLM_LAUNCH_CHECK();
  b_step_end_kernel<<<1, 32, 0, st>>>(d_step);
  UVLM_LAUNCH_CHECK();
  return ok();
}

void uvlm_batch::release() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
  void* ptrs[] = {d_cases, d_pre, d_step, d_pos_init, d_pos, d_gamma, d_gamma_prev, d_gamma_hist, d_cx, d_cy, d_cz,
                  d_normal,
                  d_area, d_uls, d_rhs, d_lx, d_ly, d_lz, d_line_uls, d_wpos, d_wpos2, d_k1, d_wgamma, d_wtx,
                  d_wty, d_wtz, d_vx, d_vy, d_vz, d_A64, d_F32, d_piv, d_tiles, d_rec, d_partial, d_in, d_plan,
                  d_totals, d_status, d_sweeps, d_res, d_loads, d_has_factor, d_refac, d_solve_order};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (st) cudaStreamDestroy(st);
  st = nullptr;
}

extern "C" {

int uvlm_batch_config_default(uvlm_batch_config* c) {
  if (!c) return UVLM_ERR_INVALID;
  *c = uvlm_batch_config{};
  c->precision = UVLM_PRECISION_MIXED;
  c->advection = UVLM_ADVECT_EULER;
  c->rk_ignore_rows = 5;
  c->refine_max_iter = 10;
  c->refine_tol = 1e-12;
  c->max_steps = 151;
  c->device = 0;
  c->use_graph = 1;
  c->stale_factors = 1;
  c->nbody_tile = -1;
  return UVLM_OK;
}

const char* uvlm_batch_nbody_tile_name(const uvlm_batch* b) {
  return b ? nbody_batch_tile_name(b->prec(), b->nb_grids.tile) : "?";
}

int uvlm_batch_create(const uvlm_batch_config* cfg, const uvlm_batch_case* cases, int32_t n_cases,
                      uvlm_batch** out) {
  if (!cfg || !cases || !out || n_cases < 1) {
    set_global_error("uvlm_batch_create: NULL argument or no cases");
    return UVLM_ERR_INVALID;
  }
  *out = nullptr;
  if ((cfg->precision != UVLM_PRECISION_FP64 && cfg->precision != UVLM_PRECISION_MIXED) ||
      (cfg->advection != UVLM_ADVECT_EULER && cfg->advection != UVLM_ADVECT_RK2) || cfg->max_steps < 1 ||
      cfg->refine_max_iter < 0 || !(cfg->refine_tol > 0) || cfg->nbody_tile < -1 ||
      cfg->nbody_tile >= kNumBatchTilesF) {
    set_global_error("uvlm_batch_create: invalid configuration (precision, advection Euler/RK2, max_steps)");
    return UVLM_ERR_INVALID;
  }
  for (int c = 0; c < n_cases; ++c) {
    const uvlm_batch_case& u = cases[c];
    if (u.rows < 1 || u.cols < 2 || (u.cols & 1) || u.rows > 64 || u.cols > 64 || u.rows * u.cols > 1024 ||
        !(u.chord > 0) ||
        !(u.span > 0) || !(u.dt > 0)) {
      set_global_error("uvlm_batch_create: every case needs 1 <= rows <= 64, even 2 <= cols <= 64, "
                            "rows * cols <= 1024, positive chord, span and dt");
      return UVLM_ERR_INVALID;
    }
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_global_error("no CUDA device");
    return UVLM_ERR_CUDA;
  }
  auto* b = new uvlm_batch();
  b->cfg = *cfg;
  b->n = n_cases;
  cudaSetDevice(cfg->device);
  cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, cfg->device);
  Error e{};
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) e = fail(kErrCuda, "stream");
  if (!e.code) e = b->alloc(cases);
  if (!e.code) e = b->tune_tiles();
  if (e.code) {
    set_global_error(e.msg);
    b->release();
    delete b;
    return e.code;
  }
  *out = b;
  return UVLM_OK;
}

int uvlm_batch_destroy(uvlm_batch* b) {
  if (!b) return UVLM_OK;
  cudaSetDevice(b->cfg.device);
  if (b->st) cudaStreamSynchronize(b->st);
  b->release();
  delete b;
  return UVLM_OK;
}

const char* uvlm_batch_last_error(const uvlm_batch* b) { return b ? b->err.c_str() : ""; }

int uvlm_batch_run(uvlm_batch* b, int64_t n_steps) {
  if (!b) return UVLM_ERR_INVALID;
  if (n_steps < 0 || b->steps_done + n_steps > b->cfg.max_steps)
    return b->fail_with(fail(kErrCapacity, "more steps than max_steps"));
  cudaSetDevice(b->cfg.device);
  for (int64_t k = 0; k < n_steps; ++k) {
    if (b->cfg.use_graph) {
      if (!b->exec) {
        const long long l0 = uvlm_kernel_launch_count();
        if (cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
          return b->fail_with(fail(kErrCuda, "graph capture could not start"));
        const Error e = b->enqueue_step();
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->st, &g);
        if (e.code) {
          if (g) cudaGraphDestroy(g);
          return b->fail_with(e);
        }
        if (ce != cudaSuccess) return b->fail_with(fail(kErrCuda, cudaGetErrorString(ce)));
        b->graph = g;
        if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess)
          return b->fail_with(fail(kErrCuda, "graph instantiation failed"));
        b->launches_per_step = uvlm_kernel_launch_count() - l0;
      }
      if (cudaGraphLaunch(b->exec, b->st) != cudaSuccess) return b->fail_with(fail(kErrCuda, "graph launch failed"));
      note_launch((int)b->launches_per_step);
    } else {
      const long long l0 = uvlm_kernel_launch_count();
      const Error e = b->enqueue_step();
      if (e.code) return b->fail_with(e);
      b->launches_per_step = uvlm_kernel_launch_count() - l0;
    }
    b->steps_done += 1;
  }
  if (cudaStreamSynchronize(b->st) != cudaSuccess) return b->fail_with(fail(kErrCuda, "batch step failed"));
  int h[4] = {0, 0, 0, 0};
  if (cudaMemcpy(h, b->d_status, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
    return b->fail_with(fail(kErrCuda, "status read failed"));
  if (h[0]) return b->fail_with(fail(kErrCapacity, "batched N-body partial buffer too small"));
  if (h[1]) return b->fail_with(fail(kErrSingular, "zero pivot in a batched LU"));
  if (h[2]) return b->fail_with(fail(kErrNonFinite, "non-finite circulation in the batch"));
  if (h[3]) return b->fail_with(fail(kErrNonFinite, "FP64 refinement did not reach the tolerance"));
  return UVLM_OK;
}

int uvlm_batch_steps_done(const uvlm_batch* b, int64_t* steps) {
  if (!b || !steps) return UVLM_ERR_INVALID;
  *steps = b->steps_done;
  return UVLM_OK;
}

int uvlm_batch_get_loads(const uvlm_batch* b, double* rows) {
  if (!b || !rows) return UVLM_ERR_INVALID;
  if (cudaMemcpy(rows, b->d_loads, sizeof(double) * 3 * (size_t)b->n * b->steps_done, cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return UVLM_ERR_CUDA;
  return UVLM_OK;
}

int uvlm_batch_get_case(const uvlm_batch* b, int32_t c, double* wing_pos, double* wing_gamma, double* wake_pos,
                        double* wake_gamma, int64_t* wake_rows) {
  if (!b || c < 0 || c >= b->n) return UVLM_ERR_INVALID;
  const BCase& k = b->hc[c];
  const long long s = b->steps_done - 1;  // the last MainLoop
  const long long rows = b->steps_done > 0 ? s : 0;
  const long long start = b->cap - 1 - std::max<long long>(s, 0);
  auto get = [](void* dst, const void* src, size_t bytes) {
    return bytes == 0 || cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
  };
  bool okk = true;
  if (wing_pos) okk &= get(wing_pos, b->d_pos + 3 * k.node_off, sizeof(double) * 3 * (k.R + 1) * (k.C + 1));
  if (wing_gamma) okk &= get(wing_gamma, b->d_gamma + k.ring_off, sizeof(double) * k.N);
  if (wake_pos && b->steps_done > 0)
    okk &= get(wake_pos, b->d_wpos + 3 * (k.wnode_off + start * (k.C + 1)), sizeof(double) * 3 * (rows + 1) * (k.C + 1));
  if (wake_gamma) okk &= get(wake_gamma, b->d_wgamma + k.wring_off + start * k.C, sizeof(double) * rows * k.C);
  if (wake_rows) *wake_rows = rows;
  return okk ? UVLM_OK : UVLM_ERR_CUDA;
}

int uvlm_batch_get_solve_stats(const uvlm_batch* b, int32_t* sweeps, double* residual) {
  if (!b) return UVLM_ERR_INVALID;
  if (sweeps && cudaMemcpy(sweeps, b->d_sweeps, sizeof(int) * b->n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return UVLM_ERR_CUDA;
  if (residual && cudaMemcpy(residual, b->d_res, sizeof(double) * b->n, cudaMemcpyDeviceToHost) != cudaSuccess)
    return UVLM_ERR_CUDA;
  return UVLM_OK;
}

int uvlm_batch_factorizations(const uvlm_batch* b, int64_t* count) {
  if (!b || !count) return UVLM_ERR_INVALID;
  unsigned long long v = 0;
  if (cudaMemcpy(&v, b->d_refac, sizeof(v), cudaMemcpyDeviceToHost) != cudaSuccess) return UVLM_ERR_CUDA;
  *count = (int64_t)v;
  return UVLM_OK;
}

int uvlm_batch_launches_per_step(const uvlm_batch* b, int64_t* launches) {
  if (!b || !launches) return UVLM_ERR_INVALID;
  *launches = b->launches_per_step;
  return UVLM_OK;
}

void* uvlm_batch_stream(const uvlm_batch* b) { return b ? (void*)b->st : nullptr; }

}  // extern "C"
