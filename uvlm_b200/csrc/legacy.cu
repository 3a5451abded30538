// legacy.cu -- C-ABI entry points of the reference's legacy (AoS
// VortexContainer) path: Morphing::Perfome / Velocity for point sets, and the
// two container load formulations, CalcLoadKatzPlotkin
// (src/calc_load/katz_plotkin.cpp:16-68) and the container form of
// CalcLoadJoukowski (src/calc_load/joukowski.h:24-104).  Rings are AoS, 12
// doubles each (VortexRing::nodes() n0..n3); a container is rows x cols
// rings, ring (i, j) at i * cols + j (VortexContainer::Index,
// src/vortex_container.h:58-60).  All arithmetic is FP64; the panel sums are
// reduced by one CTA in a fixed order.
#include <cmath>

#include "../../include/uvlm_b200.h"
#include "refapi_util.cuh"
#include "step_math.cuh"

using namespace uvlm;

namespace {

__global__ void perfome_kernel(uvlm_kinematics k, const double* __restrict__ x0, long long n, double t, int velocity,
                               double* __restrict__ out) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const d3 x = ld3(x0 + 3 * q);
    st3(out + 3 * q, velocity ? morph_velocity(k, x, t) : perfome(k, x, t));
  }
}

// Ring helpers (src/vortex.cpp): Normal :82-87, Tangent :89-94, Centroid
// :98-104, AngleOfAttack :118-122, CalcC :124-126, CalcB :128-130.
struct RingG {
  d3 n[4];
  __device__ explicit RingG(const double* r) {
#pragma unroll
    for (int q = 0; q < 4; ++q) n[q] = ld3(r + 3 * q);
  }
  __device__ d3 normal() const { return normalized(cross(sub(n[1], n[3]), sub(n[2], n[0]))); }
  __device__ d3 tangent() const { return normalized(add(sub(n[1], n[3]), sub(n[2], n[0]))); }
  __device__ d3 centroid() const { return dvs(add(add(add(n[0], n[1]), n[2]), n[3]), 4); }
  __device__ double calc_c() const { return norm(sub(n[0], n[1])); }
  __device__ double calc_b() const { return norm(sub(n[0], n[3])); }
};

__global__ void centroids_kernel(const double* __restrict__ rings, long long n, double* __restrict__ cen) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    st3(cen + 3 * q, RingG(rings + 12 * q).centroid());
}

// Segment midpoints in ForEachSegment order (src/vortex.h:132-140: start =
// nodes[k+1], end = nodes[k]).
__global__ void midpoints_kernel(const double* __restrict__ rings, long long n, double* __restrict__ t) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < 4 * n; q += (long long)gridDim.x * blockDim.x) {
    const double* r = rings + 12 * (q / 4);
    const int k = (int)(q % 4);
    st3(t + 3 * q, dvs(add(ld3(r + 3 * ((k + 1) % 4)), ld3(r + 3 * k)), 2));
  }
}

// One panel of CalcLoadKatzPlotkin: dF (3) and the Pin term, into row k of
// `terms` (4 doubles).  uw / ubc: wake and chordwise-bound velocities at the
// centroids (NULL: zero, the empty UVLMVortexRing of the legacy simulator).
__global__ void katz_plotkin_kernel(const double* __restrict__ rings, const double* __restrict__ g,
                                    const double* __restrict__ gp, int rows, int cols, uvlm_kinematics kin, d3 fs,
                                    double rho, double t, double dt, const double* __restrict__ uw,
                                    const double* __restrict__ ubc, double* __restrict__ terms) {
  const int n = rows * cols;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k / cols;
    const RingG v(rings + 12 * k);
    const d3 c = v.centroid();
    const double db = v.calc_b(), dc = v.calc_c();
    const d3 Um = sub(fs, morph_velocity(kin, c, t));  // CalcUm (functions.h:24-31)
    const d3 uh = normalized(Um);
    const d3 nr = v.normal(), tg = v.tangent();
    const double alpha = atan2(dot(Um, nr), dot(Um, tg));
    const d3 Uw = uw ? ld3(uw + 3 * k) : mk(0, 0, 0);
    const d3 Ubc = ubc ? ld3(ubc + 3 * k) : mk(0, 0, 0);
    const double dg = g[k] - (i == 0 ? 0.0 : g[k - cols]);  // DeltaGamma (vortex_container.h:87-91)
    const d3 grad = scl(tg, dg / dc);                      // Grad (vortex_container.h:93-96)
    const d3 Pn = sub(nr, scl(uh, dot(uh, nr)));            // (I - u u^T) n
    const double Lst = rho * dot(add(Um, Uw), grad) * db * dc * cos(alpha);
    const double Dst = rho * (-dot(add(Um, Ubc), Pn) * dg * db);
    double dgdt = (g[k] - gp[k]) / dt;
    if (i > 0) dgdt += (g[k - cols] - gp[k - cols]) / dt;
    dgdt /= 2;
    const double Lunst = rho * dgdt * db * dc * cos(alpha);
    const double Dunst = rho * dgdt * db * dc * sin(alpha);
    const d3 dF = add(scl(dvs(Um, norm(Um)), Dst + Dunst), scl(Pn, Lst + Lunst));
    double* o = terms + 4 * (long long)k;
    o[0] = dF.x;
    o[1] = dF.y;
    o[2] = dF.z;
    o[3] = -dot(Um, nr) * dot(dF, nr);
  }
}

// One panel of the container CalcLoadJoukowski: steady part over the panel's
// segments (the trailing-edge segment of the last row skipped) with U =
// u_ind(mid) + freestream - Vls(mid0), unsteady part Normal rho dG/dt B C,
// and the Pin term dF . Vls(reference centroid).  u: induced velocity at the
// 4 midpoints of every panel (AoS, 12 per panel).
__global__ void joukowski_kernel(const double* __restrict__ rings, const double* __restrict__ rings0,
                                 const double* __restrict__ g, const double* __restrict__ gp, int rows, int cols,
                                 uvlm_kinematics kin, d3 fs, double rho, double t, double dt,
                                 const double* __restrict__ u, double* __restrict__ terms) {
  const int n = rows * cols;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int i = k / cols;
    const bool edge = i + 1 == rows;
    const RingG v(rings + 12 * k), v0(rings0 + 12 * k);
    d3 st = mk(0, 0, 0);
    for (int q = 0; q < 4; ++q) {
      if (edge && q == 1) continue;  // trailing edge (joukowski.h:37)
      const d3 a = v.n[(q + 1) % 4], b = v.n[q];
      const d3 mid0 = dvs(add(v0.n[(q + 1) % 4], v0.n[q]), 2);
      const d3 U = add(ld3(u + 12 * (long long)k + 3 * q), sub(fs, morph_velocity(kin, mid0, t)));
      st = add(st, scl(cross(U, sub(b, a)), rho * g[k]));
    }
    const d3 un = scl(v.normal(), rho * (g[k] - gp[k]) / dt * v.calc_b() * v.calc_c());
    const d3 dF = add(st, un);
    const d3 vls = morph_velocity(kin, v0.centroid(), t);
    double* o = terms + 4 * (long long)k;
    o[0] = dF.x;
    o[1] = dF.y;
    o[2] = dF.z;
    o[3] = dot(dF, vls);
  }
}

// out[c] = sum_k a[4k + c], c < 4, in a fixed order (one CTA).
__global__ void __launch_bounds__(kSumThreads) sum4_kernel(const double* __restrict__ a, long long n, double* out) {
  __shared__ double sh[4 * kSumThreads / 32];
  double acc[4] = {0, 0, 0, 0};
  for (long long k = threadIdx.x; k < n; k += kSumThreads)
    for (int c = 0; c < 4; ++c) acc[c] += a[4 * k + c];
  for (int c = 0; c < 4; ++c)
    for (int off = 16; off; off >>= 1) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int c = 0; c < 4; ++c) sh[4 * wid + c] = acc[c];
  __syncthreads();
  if (threadIdx.x < 4) {
    double r = 0;
    for (int w = 0; w < kSumThreads / 32; ++w) r += sh[4 * w + threadIdx.x];
    out[threadIdx.x] = r;
  }
}

// Velocity induced by AoS rings at device targets (FP64), SoA -> AoS.
Error rings_velocity(const double* d_rings, const double* d_gamma, long long n_rings, int chordwise_only,
                     const double* d_targets, long long nt, double* d_out, Scratch& S) {
  double *pos, *gam, *vx, *vy, *vz;
  UVLM_TRY(S.get(&vx, nt));
  UVLM_TRY(S.get(&vy, nt));
  UVLM_TRY(S.get(&vz, nt));
  if (n_rings > 0) {
    UVLM_TRY(S.get(&pos, 12 * n_rings));
    UVLM_TRY(S.get(&gam, n_rings));
    rings_to_sheets<<<gfor(n_rings), 256>>>(d_rings, d_gamma, n_rings, pos, gam);
    UVLM_LAUNCH_CHECK();
    SheetView v{pos, 2, 0, gam, 1, 0, (int)n_rings, 2, 1, chordwise_only ? 1 : 0};
    UVLM_TRY(velocity_at(&v, 1, kNBodyFP64, d_targets, nt, vx, vy, vz, S));
  } else {
    UVLM_CUDA_TRY(cudaMemset(vx, 0, 8 * nt));
    UVLM_CUDA_TRY(cudaMemset(vy, 0, 8 * nt));
    UVLM_CUDA_TRY(cudaMemset(vz, 0, 8 * nt));
  }
  soa_to_aos<<<gfor(nt), 256>>>(vx, vy, vz, nt, d_out, nullptr, nullptr, 1.0);
  UVLM_LAUNCH_CHECK();
  return ok();
}

}  // namespace

extern "C" {

int uvlm_kinematics_perfome(const uvlm_kinematics* kin, const double* x0, int64_t n, double t, double* out) {
  if (!kin || n < 0 || (n && (!x0 || !out))) return report(fail(kErrInvalid, "invalid argument"));
  if (n == 0) return UVLM_OK;
  Scratch S;
  auto run = [&]() -> Error {
    double *dx, *dout;
    UVLM_TRY(S.up(&dx, x0, (size_t)(3 * n)));
    UVLM_TRY(S.get(&dout, (size_t)(3 * n)));
    perfome_kernel<<<gfor(n), 256>>>(*kin, dx, n, t, 0, dout);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(out, dout, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_kinematics_velocity(const uvlm_kinematics* kin, const double* x0, int64_t n, double t, double* out) {
  if (!kin || n < 0 || (n && (!x0 || !out))) return report(fail(kErrInvalid, "invalid argument"));
  if (n == 0) return UVLM_OK;
  Scratch S;
  auto run = [&]() -> Error {
    double *dx, *dout;
    UVLM_TRY(S.up(&dx, x0, (size_t)(3 * n)));
    UVLM_TRY(S.get(&dout, (size_t)(3 * n)));
    perfome_kernel<<<gfor(n), 256>>>(*kin, dx, n, t, 1, dout);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(out, dout, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_rings_load_katz_plotkin(const double* rings, const double* gamma, const double* gamma_prev, int64_t rows,
                                 int64_t cols, const uvlm_kinematics* kin, const double* bound_rings,
                                 const double* bound_gamma, int64_t n_bound, const double* wake_rings,
                                 const double* wake_gamma, int64_t n_wake, const double freestream[3], double rho,
                                 double t, double dt, double out[5]) {
  if (!rings || !gamma || !gamma_prev || rows < 1 || cols < 1 || !kin || !freestream || !out || n_bound < 0 ||
      n_wake < 0 || (n_bound && (!bound_rings || !bound_gamma)) || (n_wake && (!wake_rings || !wake_gamma)) ||
      rows * cols > (int64_t)1 << 30 || dt == 0)
    return report(fail(kErrInvalid, "invalid argument"));
  Scratch S;
  auto run = [&]() -> Error {
    const long long n = rows * cols;
    double *dr, *dg, *dgp, *cen, *uw = nullptr, *ubc = nullptr, *terms, *dout;
    UVLM_TRY(S.up(&dr, rings, (size_t)(12 * n)));
    UVLM_TRY(S.up(&dg, gamma, (size_t)n));
    UVLM_TRY(S.up(&dgp, gamma_prev, (size_t)n));
    UVLM_TRY(S.get(&cen, (size_t)(3 * n)));
    UVLM_TRY(S.get(&terms, (size_t)(4 * n)));
    UVLM_TRY(S.get(&dout, 4));
    centroids_kernel<<<gfor(n), 256>>>(dr, n, cen);
    UVLM_LAUNCH_CHECK();
    if (n_wake > 0) {  // UVLMVortexRing::InducedVelocityByWake (uvlm_vortex_ring.h:75-78)
      double *dw, *dwg;
      UVLM_TRY(S.up(&dw, wake_rings, (size_t)(12 * n_wake)));
      UVLM_TRY(S.up(&dwg, wake_gamma, (size_t)n_wake));
      UVLM_TRY(S.get(&uw, (size_t)(3 * n)));
      UVLM_TRY(rings_velocity(dw, dwg, n_wake, 0, cen, n, uw, S));
    }
    if (n_bound > 0) {  // InducedVelocityByChordwiseBound (uvlm_vortex_ring.h:80-83)
      double *db, *dbg;
      UVLM_TRY(S.up(&db, bound_rings, (size_t)(12 * n_bound)));
      UVLM_TRY(S.up(&dbg, bound_gamma, (size_t)n_bound));
      UVLM_TRY(S.get(&ubc, (size_t)(3 * n)));
      UVLM_TRY(rings_velocity(db, dbg, n_bound, 1, cen, n, ubc, S));
    }
    katz_plotkin_kernel<<<gfor(n), 256>>>(dr, dg, dgp, (int)rows, (int)cols, *kin,
                                          mk(freestream[0], freestream[1], freestream[2]), rho, t, dt, uw, ubc,
                                          terms);
    UVLM_LAUNCH_CHECK();
    sum4_kernel<<<1, kSumThreads>>>(terms, n, dout);
    UVLM_LAUNCH_CHECK();
    double r[4];
    UVLM_CUDA_TRY(cudaMemcpy(r, dout, sizeof(r), cudaMemcpyDeviceToHost));
    out[0] = r[0];
    out[1] = r[1];
    out[2] = r[2];
    out[3] = r[3];
    out[4] = 0.0;  // Pout is never accumulated (katz_plotkin.cpp:24, 66)
    return ok();
  };
  return report(run());
}

int uvlm_rings_load_joukowski(const double* rings, const double* rings0, const double* gamma,
                              const double* gamma_prev, int64_t rows, int64_t cols, const uvlm_kinematics* kin,
                              const double* vortices, const double* vortex_gamma, int64_t n_vortices,
                              const double freestream[3], double rho, double t, double dt, double out[5]) {
  if (!rings || !rings0 || !gamma || !gamma_prev || rows < 1 || cols < 1 || !kin || !freestream || !out ||
      n_vortices < 0 || (n_vortices && (!vortices || !vortex_gamma)) || rows * cols > (int64_t)1 << 28 || dt == 0)
    return report(fail(kErrInvalid, "invalid argument"));
  Scratch S;
  auto run = [&]() -> Error {
    const long long n = rows * cols;
    double *dr, *dr0, *dg, *dgp, *mid, *u, *terms, *dout;
    UVLM_TRY(S.up(&dr, rings, (size_t)(12 * n)));
    UVLM_TRY(S.up(&dr0, rings0, (size_t)(12 * n)));
    UVLM_TRY(S.up(&dg, gamma, (size_t)n));
    UVLM_TRY(S.up(&dgp, gamma_prev, (size_t)n));
    UVLM_TRY(S.get(&mid, (size_t)(12 * n)));
    UVLM_TRY(S.get(&u, (size_t)(12 * n)));
    UVLM_TRY(S.get(&terms, (size_t)(4 * n)));
    UVLM_TRY(S.get(&dout, 4));
    midpoints_kernel<<<gfor(4 * n), 256>>>(dr, n, mid);
    UVLM_LAUNCH_CHECK();
    double *dv = nullptr, *dvg = nullptr;
    if (n_vortices > 0) {
      UVLM_TRY(S.up(&dv, vortices, (size_t)(12 * n_vortices)));
      UVLM_TRY(S.up(&dvg, vortex_gamma, (size_t)n_vortices));
    }
    UVLM_TRY(rings_velocity(dv, dvg, n_vortices, 0, mid, 4 * n, u, S));
    joukowski_kernel<<<gfor(n), 256>>>(dr, dr0, dg, dgp, (int)rows, (int)cols, *kin,
                                       mk(freestream[0], freestream[1], freestream[2]), rho, t, dt, u, terms);
    UVLM_LAUNCH_CHECK();
    sum4_kernel<<<1, kSumThreads>>>(terms, n, dout);
    UVLM_LAUNCH_CHECK();
    double r[4];
    UVLM_CUDA_TRY(cudaMemcpy(r, dout, sizeof(r), cudaMemcpyDeviceToHost));
    out[0] = r[0];
    out[1] = r[1];
    out[2] = r[2];
    out[3] = r[3];
    out[4] = -r[0] * std::sqrt(freestream[0] * freestream[0] + freestream[1] * freestream[1] +
                               freestream[2] * freestream[2]);  // Pout = -Fx |U| (joukowski.h:102)
    return ok();
  };
  return report(run());
}

}  // extern "C"
