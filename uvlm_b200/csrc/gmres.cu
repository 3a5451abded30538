// gmres.cu -- FP64 GMRES(m) with an FP32 LU preconditioner.
#include <cmath>
#include <vector>

#include "gmres.cuh"

namespace uvlm {
namespace {

// y = A x (warp per row, FP64 accumulation); optionally r = b - A x.
template <class T>
__global__ void __launch_bounds__(256) matvec_kernel(const T* __restrict__ A, int n, const double* __restrict__ x,
                                                     const double* __restrict__ b, double* __restrict__ y) {
  const int lane = threadIdx.x & 31;
  const int row = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (row >= n) return;
  const T* a = A + (long long)row * n;
  double s = 0;
  if constexpr (sizeof(T) == 4) {
    // 4 floats per lane per step (16 B loads); rows start 16-byte aligned
    // only when n is a multiple of 4, otherwise scalar loads throughout
    const int n4 = (n & 3) ? 0 : n;
    for (int c = lane * 4; c < n4; c += 128) {
      const float4 v = *reinterpret_cast<const float4*>(a + c);
      s += (double)v.x * x[c] + (double)v.y * x[c + 1] + (double)v.z * x[c + 2] + (double)v.w * x[c + 3];
    }
    for (int c = n4 + lane; c < n; c += 32) s += (double)a[c] * x[c];
  } else {
    for (int c = lane; c < n; c += 32) s += a[c] * x[c];
  }
  for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (lane == 0) y[row] = b ? b[row] - s : s;
}

// h[i] = V_i . w for i <= j (one CTA per dot).
__global__ void __launch_bounds__(256) multidot_kernel(const double* V, int n, const double* w, double* h) {
  __shared__ double sh[8];
  const double* v = V + (long long)blockIdx.x * n;
  double s = 0;
  for (int k = threadIdx.x; k < n; k += 256) s += v[k] * w[k];
  for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < 8 ? sh[threadIdx.x] : 0.0;
    for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (threadIdx.x == 0) h[blockIdx.x] = s;
  }
}

// w -= sum_i h[i] V_i
__global__ void orth_kernel(const double* V, int n, int cnt, const double* h, double* w) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double s = w[k];
    for (int i = 0; i < cnt; ++i) s -= h[i] * V[(long long)i * n + k];
    w[k] = s;
  }
}

__global__ void scale_kernel(const double* src, int n, const double* hnorm, double* dst) {
  const double inv = 1.0 / hnorm[0];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) dst[k] = src[k] * inv;
}

// x += sum_i y[i] Z_i
__global__ void update_kernel(const double* Z, int n, int cnt, const double* y, double* x) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double s = x[k];
    for (int i = 0; i < cnt; ++i) s += y[i] * Z[(long long)i * n + k];
    x[k] = s;
  }
}

// y[i] = x[perm[i]]
__global__ void gather_kernel(const double* __restrict__ x, const int* __restrict__ perm, int n, double* y) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) y[k] = x[perm[k]];
}

inline int grid_n(int n) { return std::max(1, std::min(ceil_div(n, 256), 1184)); }

}  // namespace

Error matvec(const float* A32, const double* A64, int n, const double* x, double* y, cudaStream_t st) {
  if (A32)
    matvec_kernel<float><<<ceil_div(n, 8), 256, 0, st>>>(A32, n, x, nullptr, y);
  else
    matvec_kernel<double><<<ceil_div(n, 8), 256, 0, st>>>(A64, n, x, nullptr, y);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error gmres_work_alloc(GmresWork* g, int n, int m) {
  gmres_work_free(g);
  g->n = n;
  g->m = m;
  UVLM_CUDA_TRY(cudaMalloc(&g->V, sizeof(double) * (size_t)(m + 1) * n));
  UVLM_CUDA_TRY(cudaMalloc(&g->Z, sizeof(double) * (size_t)m * n));
  UVLM_CUDA_TRY(cudaMalloc(&g->w, sizeof(double) * n));
  UVLM_CUDA_TRY(cudaMalloc(&g->h, sizeof(double) * 2 * (m + 2)));
  UVLM_CUDA_TRY(cudaMalloc(&g->y, sizeof(double) * (m + 1)));
  UVLM_CUDA_TRY(cudaMalloc(&g->ptmp, sizeof(float) * 2 * n));
  UVLM_CUDA_TRY(cudaMallocHost(&g->hh, sizeof(double) * 2 * (m + 2)));
  return ok();
}

void gmres_work_free(GmresWork* g) {
  cudaFree(g->V);
  cudaFree(g->Z);
  cudaFree(g->w);
  cudaFree(g->h);
  cudaFree(g->y);
  cudaFree(g->ptmp);
  if (g->hh) cudaFreeHost(g->hh);
  *g = GmresWork{};
}

Error gmres_solve(const float* A32, const double* A64, int n, const float* LU, LuWork* lu, const float* Minv,
                  const double* b, double* x, double tol, int max_iter, GmresWork* g, GmresResult* res,
                  cudaStream_t st) {
  const int m = g->m;
  res->iters = 0;
  res->converged = false;
  res->nonfinite_guess = false;
  auto matvec_res = [&](const double* xin, double* out) -> Error {
    if (A32)
      matvec_kernel<float><<<ceil_div(n, 8), 256, 0, st>>>(A32, n, xin, b, out);
    else
      matvec_kernel<double><<<ceil_div(n, 8), 256, 0, st>>>(A64, n, xin, b, out);
    UVLM_LAUNCH_CHECK();
    return ok();
  };
  auto norm2 = [&](const double* v, double* out_host) -> Error {
    multidot_kernel<<<1, 256, 0, st>>>(v, n, v, g->h + m + 1);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpyAsync(out_host, g->h + m + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    UVLM_CUDA_TRY(cudaStreamSynchronize(st));
    *out_host = std::sqrt(*out_host);
    return ok();
  };
  double bnorm = 0;
  UVLM_TRY(norm2(b, &bnorm));
  if (!std::isfinite(bnorm)) return fail(kErrNonFinite, "non-finite right-hand side");
  if (!(bnorm > 0)) {
    UVLM_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    res->converged = true;
    res->relres = 0;
    return ok();
  }
  std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), gv(m + 1), yv(m);
  int total = 0;
  while (true) {
    // r0 = b - A x  -> V_0
    UVLM_TRY(matvec_res(x, g->V));
    double beta = 0;
    UVLM_TRY(norm2(g->V, &beta));
    res->relres = beta / bnorm;
    if (total == 0) res->initial_relres = res->relres;
    if (!std::isfinite(beta)) {
      // a non-finite initial guess (the RHS is finite): not converged, so the
      // caller can take its fallback; later it is an error of the iteration
      if (total == 0) {
        res->converged = false;
        res->nonfinite_guess = true;
        return ok();
      }
      return fail(kErrNonFinite, "non-finite GMRES residual");
    }
    if (beta <= tol * bnorm) {
      res->converged = true;
      break;
    }
    if (total >= max_iter) break;
    {
      double* hb = g->h + m + 1;
      g->hh[0] = beta;
      UVLM_CUDA_TRY(cudaMemcpyAsync(hb, g->hh, sizeof(double), cudaMemcpyHostToDevice, st));
      scale_kernel<<<grid_n(n), 256, 0, st>>>(g->V, n, hb, g->V);
      UVLM_LAUNCH_CHECK();
    }
    std::fill(gv.begin(), gv.end(), 0.0);
    gv[0] = beta;
    int j = 0;
    for (; j < m && total < max_iter; ++j) {
      double* Vj = g->V + (size_t)j * n;
      double* Zj = g->Z + (size_t)j * n;
      if (Minv) {
        // Z_j = (LU)^-1 P V_j: the row permutation of the factors, then the dense inverse
        gather_kernel<<<grid_n(n), 256, 0, st>>>(Vj, lu->ipiv + n, n, g->w);
        UVLM_LAUNCH_CHECK();
        UVLM_TRY(matvec(Minv, nullptr, n, g->w, Zj, st));
      } else
        UVLM_TRY(lu_solve_f32(LU, n, lu, Vj, Zj, g->ptmp, st));
      UVLM_TRY(matvec(A32, A64, n, Zj, g->w, st));
      // classical Gram-Schmidt, applied twice (CGS2)
      for (int pass = 0; pass < 2; ++pass) {
        multidot_kernel<<<j + 1, 256, 0, st>>>(g->V, n, g->w, g->h + pass * (m + 2));
        UVLM_LAUNCH_CHECK();
        orth_kernel<<<grid_n(n), 256, 0, st>>>(g->V, n, j + 1, g->h + pass * (m + 2), g->w);
        UVLM_LAUNCH_CHECK();
      }
      multidot_kernel<<<1, 256, 0, st>>>(g->w, n, g->w, g->h + m + 1);
      UVLM_LAUNCH_CHECK();
      UVLM_CUDA_TRY(cudaMemcpyAsync(g->hh, g->h, sizeof(double) * 2 * (m + 2), cudaMemcpyDeviceToHost, st));
      UVLM_CUDA_TRY(cudaStreamSynchronize(st));
      const double hnext = std::sqrt(g->hh[m + 1]);
      for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = g->hh[i] + g->hh[(m + 2) + i];
      H[(size_t)(j + 1) * m + j] = hnext;
      // V_{j+1} = w / hnext
      g->hh[0] = hnext;
      UVLM_CUDA_TRY(cudaMemcpyAsync(g->h + m + 1, g->hh, sizeof(double), cudaMemcpyHostToDevice, st));
      scale_kernel<<<grid_n(n), 256, 0, st>>>(g->w, n, g->h + m + 1, g->V + (size_t)(j + 1) * n);
      UVLM_LAUNCH_CHECK();
      // Givens rotations on the Hessenberg column
      for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * m + j], bb = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * bb;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * bb;
      }
      const double a = H[(size_t)j * m + j], bb = H[(size_t)(j + 1) * m + j];
      const double r = std::hypot(a, bb);
      cs[j] = r > 0 ? a / r : 1.0;
      sn[j] = r > 0 ? bb / r : 0.0;
      H[(size_t)j * m + j] = r;
      H[(size_t)(j + 1) * m + j] = 0;
      gv[j + 1] = -sn[j] * gv[j];
      gv[j] = cs[j] * gv[j];
      ++total;
      if (!std::isfinite(gv[j + 1])) return fail(kErrNonFinite, "non-finite GMRES iteration");
      if (std::fabs(gv[j + 1]) <= tol * bnorm || !(hnext > 0)) {
        ++j;
        break;
      }
    }
    // y = H^-1 g (upper triangular j x j), x += Z y
    for (int i = j - 1; i >= 0; --i) {
      double s = gv[i];
      for (int k = i + 1; k < j; ++k) s -= H[(size_t)i * m + k] * yv[k];
      yv[i] = s / H[(size_t)i * m + i];
    }
    UVLM_CUDA_TRY(cudaMemcpyAsync(g->y, yv.data(), sizeof(double) * j, cudaMemcpyHostToDevice, st));
    update_kernel<<<grid_n(n), 256, 0, st>>>(g->Z, n, j, g->y, x);
    UVLM_LAUNCH_CHECK();
  }
  res->iters = total;
  return ok();
}

}  // namespace uvlm
