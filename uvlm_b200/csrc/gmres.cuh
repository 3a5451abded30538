// gmres.cuh -- restarted, right-preconditioned GMRES with FP64 vectors and
// residuals, preconditioned by (possibly stale) FP32 LU factors.
//
// New relative to the reference (whose solve is Eigen::FullPivLU each step,
// src/simulator/simple_simulator.cpp:264-268): the mixed-precision form
// factors in TF32/BF16 only when it must and wins FP64 accuracy back through
// Krylov iterations whose residual b - A x is formed in FP64 on the GPU.
#pragma once

#include "common.cuh"
#include "lu.cuh"

namespace uvlm {

struct GmresWork {
  int n = 0, m = 0;
  double* V = nullptr;   // [m+1][n]
  double* Z = nullptr;   // [m][n]   preconditioned directions
  double* w = nullptr;   // [n]
  double* h = nullptr;   // [2][m+1] device dot products
  double* hh = nullptr;  // pinned host copy
  float* ptmp = nullptr; // [2n] preconditioner scratch
  double* y = nullptr;   // [m] device
};

struct GmresResult {
  int iters = 0;
  double relres = 0;
  double initial_relres = 0;  // ||b - A x0|| / ||b|| of the initial guess
  bool converged = false;
  bool nonfinite_guess = false;  // the initial guess gave a non-finite residual (nothing iterated)
};

Error gmres_work_alloc(GmresWork* g, int n, int m);
void gmres_work_free(GmresWork* g);

// Solves A x = b.  Exactly one of A32 / A64 is non-null (the residual matrix,
// read with FP64 accumulation).  LU/lu are FP32 factors (lu_factor_f32) of a
// nearby matrix.  Minv, when non-null, is (LU)^-1 as a dense FP32 matrix
// (lu_inverse_f32), applied after the row permutation of the factors (perm =
// lu->ipiv + n) in place of the triangular solves.  x holds the initial
// guess on entry.
Error gmres_solve(const float* A32, const double* A64, int n, const float* LU, LuWork* lu, const float* Minv,
                  const double* b, double* x, double tol, int max_iter, GmresWork* g, GmresResult* res,
                  cudaStream_t st);

// y = A x for a row-major FP32 or FP64 matrix with FP64 accumulation.
Error matvec(const float* A32, const double* A64, int n, const double* x, double* y, cudaStream_t st);

}  // namespace uvlm
