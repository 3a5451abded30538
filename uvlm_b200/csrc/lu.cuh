// lu.cuh -- blocked right-looking LU with partial pivoting and triangular
// solves on the GPU.
//
// Replaces Eigen::FullPivLU<MatrixXd>(A).solve(rhs) of
// SimpleSimulator::MainLoop (src/simulator/simple_simulator.cpp:264-268) and of
// the legacy SolveLinearProblem (src/linear.inl:125-129, :152-156).  The
// reference pivots completely; this factorisation pivots by rows (the pivot
// of each column is the largest |a| below the diagonal), which changes the
// result only at the rounding level for the influence matrices of the path.
//
// Layout: A is row-major n x n (row K = collocation point, column L = ring).
// Factor: per panel of kLuNB columns
//   1. lu_panel   -- one thread-block cluster (<= 16 CTAs of 256 rows): the
//                    pivot rows chosen by a tournament (each CTA factors its
//                    rows, candidate sets merged in a 4-ary tree through
//                    distributed shared memory), then L21 by substitution;
//                    else a cluster with one barrier per column; else one
//                    cooperative kernel with a bounded grid barrier per column;
//   2. laswp      -- the panel's row swaps applied to the other columns;
//   3. trsm       -- U12 = L11^-1 A12;
//   4. update     -- A22 -= L21 U12: FP64 SIMT GEMM (plain form) or a tcgen05
//                    tensor-core GEMM in TF32 / BF16 with FP32 accumulation
//                    (mixed form, lu_tc.cu).
// Solve: the inverses of the diagonal blocks of L and U are formed once per
// factorisation; forward/backward substitution is then one cooperative
// kernel per triangle in which block row I waits (bounded) for the solution of
// the block rows before it and applies their GEMV contributions.
#pragma once

#include "common.cuh"

namespace uvlm {

constexpr int kLuNB = 64;   // panel width
constexpr int kTriB = 64;   // triangular-solve block

enum LuUpdate { kLuUpdateSimt = 0, kLuUpdateTF32 = 1, kLuUpdateBF16 = 2 };

struct LuWork {
  int n = 0;
  int* ipiv = nullptr;        // [n]
  int* err = nullptr;         // [1]: 0 ok, 1 barrier timeout, 2 zero pivot, 3 solve timeout
  unsigned* bar = nullptr;    // [2] grid barrier state
  double* cand_val = nullptr; // [2][kMaxCtas]
  int* cand_row = nullptr;    // [2][kMaxCtas]
  void* cand_data = nullptr;  // [2][kMaxCtas][kLuNB] of the factor type
  void* diag_data = nullptr;  // [2][kLuNB]
  void* dinv_l = nullptr;     // [nblk][kTriB][kTriB] inverses of the diagonal blocks of L
  void* dinv_u = nullptr;     // [nblk][kTriB][kTriB] inverses of the diagonal blocks of U
  float* a3 = nullptr;        // [n][3 kTriB] split-TF32 operands of the dense inverse's updates
  float* b3 = nullptr;        // [n][3 kTriB]
  unsigned* flags = nullptr;  // [2][nblk] solve progress flags (epoch tagged)
  unsigned epoch = 0;
  void* ut = nullptr;         // tensor-core path: U12 transposed (K-major B operand)
  void* opA = nullptr;        // tensor-core path: BF16 copies of the operands
  void* opB = nullptr;
  int elem_size = 8;
  int num_sms = 148;
  bool tournament = true;     // panel pivots by a tournament (one cluster per panel) where it fits
  bool local_pivot = false;   // tournament panel: pivots only among each panel's top 256 rows (a
                              // preconditioner's factors; L may then exceed 1 in magnitude)
};

constexpr int kLuMaxCtas = 148;

Error lu_work_alloc(LuWork* w, int n, int elem_size, int num_sms);
void lu_work_free(LuWork* w);

// In-place factorisation PA = LU of a row-major n x n matrix.
Error lu_factor_f64(double* A, int n, LuWork* w, cudaStream_t st);
Error lu_factor_f32(float* A, int n, LuUpdate upd, LuWork* w, cudaStream_t st);
// Returns kErrSingular / kErrTimeout from the device error word (syncs).
Error lu_check(LuWork* w, cudaStream_t st);

// x = A^-1 b with the factors of lu_factor_f64 (FP64 throughout).
Error lu_solve_f64(const double* LU, int n, LuWork* w, const double* b, double* x, double* tmp, cudaStream_t st);
// z = (LU)^-1 v with FP32 factors: FP64 in/out, FP32 arithmetic (preconditioner).
Error lu_solve_f32(const float* LU, int n, LuWork* w, const double* v, double* z, float* tmp, cudaStream_t st);

// X = (LU)^-1 = U^-1 L^-1 as a dense row-major FP32 matrix from the factors
// of lu_factor_f32 (block forward then backward substitution on the identity,
// GEMM updates between the diagonal-block inverses; the forward pass updates
// only the lower-triangular part it can fill).  A^-1 = X P: applied to v as
// X (P v) with (P v)[i] = v[perm[i]], perm = ipiv + n of the same LuWork.
// A stale preconditioner applied as one gather and one dense matrix-vector
// product.
Error lu_inverse_f32(const float* LU, int n, LuUpdate upd, LuWork* w, float* X, cudaStream_t st);

// Trailing update used by the factorisation (exposed for tests/benches):
// C[m x nc] -= A[m x k] * B[k x nc], row-major with leading dims.
Error gemm_update_f64(double* C, int ldc, const double* A, int lda, const double* B, int ldb, int m, int nc, int k,
                      cudaStream_t st);
Error gemm_update_f32_simt(float* C, int ldc, const float* A, int lda, const float* B, int ldb, int m, int nc, int k,
                           cudaStream_t st);
// tcgen05 path (lu_tc.cu): C -= A * Bt^T with A [m x k] (lda), Bt [nc x k]
// (ldbt) K-major, k a multiple of 32 (TF32) / 64 (BF16 copies are made here).
Error gemm_update_tc(float* C, int ldc, const float* A, int lda, const float* Bt, int ldbt, int m, int nc, int k,
                     LuUpdate kind, LuWork* w, cudaStream_t st);
bool gemm_tc_available();
// The bounded-wait limit of this unit's kernels (0 = default), and a check
// that a wait on a flag nothing sets gives up after `cycles` (restores the
// default limit afterwards).
Error lu_set_wait_limit(long long cycles);
Error tc_set_wait_limit(long long cycles);
Error lu_wait_probe(long long cycles, bool* gave_up);

}  // namespace uvlm
