// refapi.cu -- context-free C-ABI replacements of the reference's API:
// UVLM::InducedVelocity (sheet and AoS-ring forms), advect::Advection,
// UVLM::AdvectParallel / ConnectTrailingEdge, UVLM::SolveLinearProblem and the
// dense FullPivLU solve.  Each call uploads its host arrays, runs the same
// kernels as the time-stepper and copies the result back.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/uvlm_b200.h"
#include "gmres.cuh"
#include "lu.cuh"
#include "nbody.cuh"
#include "refapi_util.cuh"
#include "step.cuh"

using namespace uvlm;

namespace {

__global__ void connect_te_kernel(const double* edge, long long n, double* wake) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    for (int d = 0; d < 3; ++d) {
      wake[12 * k + 0 + d] = edge[12 * k + 3 + d];  // wake.nodes[0] = edge.nodes[1]
      wake[12 * k + 9 + d] = edge[12 * k + 6 + d];  // wake.nodes[3] = edge.nodes[2]
    }
  }
}
__global__ void f64_to_f32(const double* a, long long n, float* b) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    b[k] = (float)a[k];
}
// Row-shifted copy of the previous AB2 velocity: dst row i <- src row i-1.
__global__ void shift_rows_kernel(const double* src, int num, int src_rows, double* dst, int dst_rows, int row_elems) {
  const long long total = (long long)num * dst_rows * row_elems;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(k % row_elems);
    const long long nr = k / row_elems;
    const int i = (int)(nr % dst_rows), n = (int)(nr / dst_rows);
    dst[k] = (i >= 1 && i - 1 < src_rows) ? src[((long long)n * src_rows + i - 1) * row_elems + e] : 0.0;
  }
}

// ----------------------------------------------- impulse post-processing
// Midpoints of the four segments of every panel in ForEachSegment order
// (vortex.h:132-140: start = nodes[k+1], end = nodes[k]) as AoS targets.
__global__ void lamb_midpoints_kernel(const double* __restrict__ panels, long long n, double* __restrict__ t) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < 4 * n; q += (long long)gridDim.x * blockDim.x) {
    const long long i = q / 4;
    const int k = (int)(q % 4);
    const double* p = panels + 12 * i;
    const d3 start = ld3(p + 3 * ((k + 1) % 4)), end = ld3(p + 3 * k);
    st3(t + 3 * q, dvs(add(start, end), 2));
  }
}

// CalcLambVectorOnPanel (calc_impulse.h:15-30) summed over the panels as
// calc_impulse_main.cpp:79-82 does, FP64, one CTA (fixed summation order):
// ue = v_node[k] + u(mid_k) - freestream_i, res += (ue x dl) * gamma,
// dl = end - start.
__global__ void __launch_bounds__(kSumThreads) lamb_sum_kernel(const double* __restrict__ panels,
                                                               const double* __restrict__ pg,
                                                               const double* __restrict__ vnodes,
                                                               const double* __restrict__ fs, long long n,
                                                               const double* __restrict__ u, double* out) {
  __shared__ double sh[3 * kSumThreads / 32];
  d3 acc = mk(0, 0, 0);
  for (long long i = threadIdx.x; i < n; i += kSumThreads) {
    const double* p = panels + 12 * i;
    const d3 f = ld3(fs + 3 * i);
    d3 a = mk(0, 0, 0);
    for (int k = 0; k < 4; ++k) {
      const d3 dl = sub(ld3(p + 3 * k), ld3(p + 3 * ((k + 1) % 4)));
      const d3 ue = sub(add(ld3(vnodes + 12 * i + 3 * k), ld3(u + 3 * (4 * i + k))), f);
      a = add(a, scl(cross(ue, dl), pg[i]));
    }
    acc = add(acc, a);
  }
  const d3 r = block_sum3(acc, sh);
  if (threadIdx.x == 0) st3(out, r);
}

// CalcVortexImpulse (calc_impulse_main.cpp:34-41): sum of Normal * gamma *
// Area * (-1) (vortex.cpp:140-143; Normal :82-87, Area :132-138), one CTA.
__global__ void __launch_bounds__(kSumThreads) vortex_impulse_kernel(const double* __restrict__ rings,
                                                                     const double* __restrict__ g, long long n,
                                                                     double* out) {
  __shared__ double sh[3 * kSumThreads / 32];
  d3 acc = mk(0, 0, 0);
  for (long long i = threadIdx.x; i < n; i += kSumThreads) {
    const double* r = rings + 12 * i;
    const d3 a = ld3(r), b = ld3(r + 3), c = ld3(r + 6), d = ld3(r + 9);
    const d3 nrm = normalized(cross(sub(b, d), sub(c, a)));
    const double area = (norm(cross(sub(b, a), sub(d, a))) + norm(cross(sub(d, c), sub(b, c)))) / 2;
    acc = add(acc, scl(nrm, -g[i] * area));
  }
  const d3 r = block_sum3(acc, sh);
  if (threadIdx.x == 0) st3(out, r);
}

// SolveLinearProblem over AoS rings (src/linear.inl:113-157): FP64
// assembly, RHS with ring i moving by kins[kin_of[i]] (kin_of NULL: kins[0]),
// optional wake term, FP64 LU solve.
Error solve_rings(const double* bound_rings, const double* bound_rings0, int64_t n_bound,
                  const uvlm_kinematics* kins, int n_kins, const int* kin_of, const double* wake_rings,
                  const double* wake_gamma, int64_t n_wake, const double freestream[3], double t,
                  int32_t drop_wake_term, double* gamma_out) {
  Scratch S;
  const int n = (int)n_bound;
  double *dr, *dr0, *A, *cen, *nrm, *b, *x, *tmp, *wv = nullptr;
  uvlm_kinematics* dk;
  int* dko = nullptr;
  UVLM_TRY(S.up(&dr, bound_rings, (size_t)12 * n));
  UVLM_TRY(S.up(&dr0, bound_rings0 ? bound_rings0 : bound_rings, (size_t)12 * n));
  UVLM_TRY(S.up(&dk, kins, (size_t)n_kins));
  if (kin_of) UVLM_TRY(S.up(&dko, kin_of, (size_t)n));
  UVLM_TRY(S.get(&A, (size_t)n * n));
  UVLM_TRY(S.get(&cen, (size_t)3 * n));
  UVLM_TRY(S.get(&nrm, (size_t)3 * n));
  UVLM_TRY(S.get(&b, (size_t)n));
  UVLM_TRY(S.get(&x, (size_t)n));
  UVLM_TRY(S.get(&tmp, (size_t)n));
  UVLM_TRY(launch_assemble_rings(dr, n, A, cen, nrm, 0));
  if (!drop_wake_term && n_wake > 0) {
    double *dw, *dg, *pos, *gam, *vx, *vy, *vz;
    UVLM_TRY(S.up(&dw, wake_rings, (size_t)12 * n_wake));
    UVLM_TRY(S.up(&dg, wake_gamma, (size_t)n_wake));
    UVLM_TRY(S.get(&pos, (size_t)12 * n_wake));
    UVLM_TRY(S.get(&gam, (size_t)n_wake));
    UVLM_TRY(S.get(&vx, n));
    UVLM_TRY(S.get(&vy, n));
    UVLM_TRY(S.get(&vz, n));
    UVLM_TRY(S.get(&wv, (size_t)3 * n));
    rings_to_sheets<<<gfor(n_wake), 256>>>(dw, dg, n_wake, pos, gam);
    UVLM_LAUNCH_CHECK();
    SheetView v{pos, 2, 0, gam, 1, 0, (int)n_wake, 2, 1};
    UVLM_TRY(velocity_at(&v, 1, kNBodyFP64, cen, n, vx, vy, vz, S));
    soa_to_aos<<<gfor(n), 256>>>(vx, vy, vz, n, wv, nullptr, nullptr, 1.0);
    UVLM_LAUNCH_CHECK();
  }
  UVLM_TRY(launch_legacy_rhs(dk, dko, dr0, n, cen, nrm, freestream, t, wv, b, 0));
  LuWork lu;
  UVLM_TRY(lu_work_alloc(&lu, n, 8, sms()));
  Error e = lu_factor_f64(A, n, &lu, 0);
  if (!e.code) e = lu_check(&lu, 0);
  if (!e.code) e = lu_solve_f64(A, n, &lu, b, x, tmp, 0);
  if (!e.code) e = lu_check(&lu, 0);
  lu_work_free(&lu);
  UVLM_TRY(e);
  UVLM_CUDA_TRY(cudaMemcpy(gamma_out, x, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return ok();
}

}  // namespace

struct uvlm_advection {
  int scheme = 0;
  int precision = 0;
  bool has_prev = false;
  int prev_rows = 0, prev_num = 0, prev_cols = 0;
  std::vector<double> vprev;  // logical layout of the previous call (host copy)
};

extern "C" {

int uvlm_sheet_induced_velocity(const double* pos, const double* gamma, int64_t num, int64_t grows, int64_t gcols,
                                const double* targets, int64_t n_targets, double* out, int32_t precision) {
  if (!pos || !targets || !out || (num * grows * gcols > 0 && !gamma) || num < 0 || grows < 0 || gcols < 0 ||
      n_targets < 0)
    return report(fail(kErrInvalid, "invalid argument"));
  if (n_targets == 0) return UVLM_OK;
  Scratch S;
  const NBodyPrec prec = precision == UVLM_PRECISION_MIXED ? kNBodyFP32 : kNBodyFP64;
  double *dp, *dg, *dt, *vx, *vy, *vz, *dout;
  Error e;
  auto run = [&]() -> Error {
    UVLM_TRY(S.up(&dp, pos, (size_t)(num * (grows + 1) * (gcols + 1) * 3)));
    UVLM_TRY(S.up(&dg, gamma, (size_t)(num * grows * gcols)));
    UVLM_TRY(S.up(&dt, targets, (size_t)(3 * n_targets)));
    UVLM_TRY(S.get(&vx, n_targets));
    UVLM_TRY(S.get(&vy, n_targets));
    UVLM_TRY(S.get(&vz, n_targets));
    UVLM_TRY(S.get(&dout, 3 * n_targets));
    SheetView v{dp, (int)grows + 1, 0, dg, (int)grows, 0, (int)num, (int)grows + 1, (int)gcols};
    const int nv = (grows > 0 && gcols > 0 && num > 0) ? 1 : 0;
    if (nv)
      UVLM_TRY(velocity_at(&v, nv, prec, dt, n_targets, vx, vy, vz, S));
    else {
      UVLM_CUDA_TRY(cudaMemset(vx, 0, 8 * n_targets));
      UVLM_CUDA_TRY(cudaMemset(vy, 0, 8 * n_targets));
      UVLM_CUDA_TRY(cudaMemset(vz, 0, 8 * n_targets));
    }
    soa_to_aos<<<gfor(n_targets), 256>>>(vx, vy, vz, n_targets, dout, nullptr, nullptr, 1.0);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(out, dout, sizeof(double) * 3 * n_targets, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_advection_create(const char* name, int32_t precision, uvlm_advection** out) {
  if (!name || !out) return report(fail(kErrInvalid, "NULL argument"));
  const std::string s(name);
  int a = -1;
  if (s == "euler") a = UVLM_ADVECT_EULER;
  if (s == "RK2") a = UVLM_ADVECT_RK2;
  if (s == "RK4") a = UVLM_ADVECT_RK4;
  if (s == "AB2") a = UVLM_ADVECT_AB2;
  if (a < 0) return report(fail(kErrInvalid, "Invalid advection name! Please choose from following: [AB2, RK2, RK4, euler]"));
  auto* adv = new uvlm_advection();
  adv->scheme = a;
  adv->precision = precision;
  *out = adv;
  return UVLM_OK;
}

int uvlm_advection_destroy(uvlm_advection* adv) {
  delete adv;
  return UVLM_OK;
}

int uvlm_advection_advect(uvlm_advection* adv, double* next, const double* wing_pos, const double* wing_gamma,
                          int64_t num, int64_t rows, int64_t cols, const double* wake_pos, const double* wake_gamma,
                          int64_t wake_rows, const double ff[3], double dt) {
  if (!adv || !next || !wing_pos || !wing_gamma || !wake_pos || !ff || num < 1 || rows < 1 || cols < 1 ||
      wake_rows < 0 || (wake_rows > 0 && !wake_gamma))
    return report(fail(kErrInvalid, "invalid argument"));
  Scratch S;
  const NBodyPrec prec = adv->precision == UVLM_PRECISION_MIXED ? kNBodyFP32 : kNBodyFP64;
  const int C = (int)cols, nodes = (int)wake_rows + 1;
  const size_t wn = (size_t)num * nodes * (C + 1) * 3;
  auto run = [&]() -> Error {
    double *dwing, *dwg, *x, *pos2, *k1, *k2, *k3, *vprev, *dwg2, *vx, *vy, *vz, *targets;
    UVLM_TRY(S.up(&dwing, wing_pos, (size_t)num * (rows + 1) * (cols + 1) * 3));
    UVLM_TRY(S.up(&dwg, wing_gamma, (size_t)num * rows * cols));
    UVLM_TRY(S.up(&x, wake_pos, wn));
    UVLM_TRY(S.get(&pos2, wn));
    UVLM_TRY(S.get(&k1, wn));
    UVLM_TRY(S.get(&k2, wn));
    UVLM_TRY(S.get(&k3, wn));
    UVLM_TRY(S.get(&vprev, wn));
    // wake circulation in the node-row layout (ring row i on node row i)
    std::vector<double> g((size_t)num * nodes * C, 0.0);
    for (int64_t n = 0; n < num; ++n)
      for (int64_t i = 0; i < wake_rows; ++i)
        std::memcpy(&g[((size_t)n * nodes + i) * C], wake_gamma + ((size_t)n * wake_rows + i) * C, sizeof(double) * C);
    UVLM_TRY(S.up(&dwg2, g.data(), g.size()));
    const long long nt = (long long)num * (nodes - 1) * (C + 1);
    UVLM_TRY(S.get(&vx, std::max<long long>(nt, 1)));
    UVLM_TRY(S.get(&vy, std::max<long long>(nt, 1)));
    UVLM_TRY(S.get(&vz, std::max<long long>(nt, 1)));
    UVLM_TRY(S.get(&targets, 3 * std::max<long long>(nt, 1)));
    const WakeLayout L{(int)num, C, nodes, 0, nodes};
    auto vel = [&](const double* P) -> Error {
      if (nt == 0) return ok();
      double *tx, *ty, *tz;
      UVLM_TRY(S.get(&tx, nt));
      UVLM_TRY(S.get(&ty, nt));
      UVLM_TRY(S.get(&tz, nt));
      UVLM_TRY(launch_gather_wake(L, P, tx, ty, tz, 0));
      soa_to_aos<<<gfor(nt), 256>>>(tx, ty, tz, nt, targets, nullptr, nullptr, 1.0);
      UVLM_LAUNCH_CHECK();
      SheetView views[2] = {
          SheetView{dwing, (int)rows + 1, 0, dwg, (int)rows, 0, (int)num, (int)rows + 1, C},
          SheetView{P, nodes, 0, dwg2, nodes, 0, (int)num, nodes, C}};
      const int nv = wake_rows > 0 ? 2 : 1;
      return velocity_at(views, nv, prec, targets, nt, vx, vy, vz, S);
    };
    const int ign = 5;
    switch (adv->scheme) {
      case UVLM_ADVECT_EULER:
        UVLM_TRY(vel(x));
        UVLM_TRY(launch_advect(kAdvEuler, L, x, pos2, k1, k2, k3, vprev, false, vx, vy, vz, ff, dt, ign, 0));
        break;
      case UVLM_ADVECT_RK2:
        UVLM_TRY(vel(x));
        UVLM_TRY(launch_advect(kAdvRK2K1, L, x, pos2, k1, k2, k3, vprev, false, vx, vy, vz, ff, dt, ign, 0));
        UVLM_TRY(vel(pos2));
        UVLM_TRY(launch_advect(kAdvRK2Upd, L, x, pos2, k1, k2, k3, vprev, false, vx, vy, vz, ff, dt, ign, 0));
        break;
      case UVLM_ADVECT_RK4:
        UVLM_TRY(vel(x));
        UVLM_TRY(launch_advect(kAdvRK4K1, L, x, pos2, k1, k2, k3, vprev, false, vx, vy, vz, ff, dt, ign, 0));
        UVLM_TRY(vel(pos2));
        UVLM_TRY(launch_advect(kAdvRK4K2, L, x, pos2, k1, k2, k3, vprev, false, vx, vy, vz, ff, dt, ign, 0));
        UVLM_TRY(vel(pos2));
        UVLM_TRY(launch_advect(kAdvRK4Upd, L, x, pos2, k1, k2, k3, vprev, false, vx, vy, vz, ff, dt, ign, 0));
        break;
      case UVLM_ADVECT_AB2: {
        // v_prev(n, i-1, j) of the previous call pairs with v(n, i, j)
        const bool hp = adv->has_prev && adv->prev_num == num && adv->prev_cols == C;
        if (hp) {
          double* prev;
          UVLM_TRY(S.up(&prev, adv->vprev.data(), adv->vprev.size()));
          shift_rows_kernel<<<gfor((long long)wn), 256>>>(prev, (int)num, adv->prev_rows, vprev, nodes, 3 * (C + 1));
          UVLM_LAUNCH_CHECK();
        }
        UVLM_TRY(vel(x));
        UVLM_TRY(launch_advect(kAdvAB2, L, x, pos2, k1, k2, k3, vprev, hp, vx, vy, vz, ff, dt, ign, 0));
        adv->vprev.resize(wn);
        UVLM_CUDA_TRY(cudaMemcpy(adv->vprev.data(), vprev, sizeof(double) * wn, cudaMemcpyDeviceToHost));
        adv->has_prev = true;
        adv->prev_rows = nodes;
        adv->prev_num = (int)num;
        adv->prev_cols = C;
        break;
      }
      default:
        return fail(kErrInvalid, "unknown scheme");
    }
    UVLM_CUDA_TRY(cudaMemcpy(next, x, sizeof(double) * wn, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_rings_induced_velocity(const double* rings, const double* gammas, int64_t n_rings, const double* targets,
                                int64_t n_targets, int32_t chordwise_only, double* out) {
  if (n_rings < 0 || n_targets < 0 || !out || (n_targets && !targets) || (n_rings && (!rings || !gammas)))
    return report(fail(kErrInvalid, "invalid argument"));
  if (n_targets == 0) return UVLM_OK;
  Scratch S;
  auto run = [&]() -> Error {
    double *dr, *dg, *pos, *gam, *dt, *vx, *vy, *vz, *dout;
    UVLM_TRY(S.up(&dt, targets, (size_t)(3 * n_targets)));
    UVLM_TRY(S.get(&vx, n_targets));
    UVLM_TRY(S.get(&vy, n_targets));
    UVLM_TRY(S.get(&vz, n_targets));
    UVLM_TRY(S.get(&dout, 3 * n_targets));
    if (n_rings > 0) {
      UVLM_TRY(S.up(&dr, rings, (size_t)(12 * n_rings)));
      UVLM_TRY(S.up(&dg, gammas, (size_t)n_rings));
      UVLM_TRY(S.get(&pos, 12 * n_rings));
      UVLM_TRY(S.get(&gam, n_rings));
      rings_to_sheets<<<gfor(n_rings), 256>>>(dr, dg, n_rings, pos, gam);
      UVLM_LAUNCH_CHECK();
      SheetView v{pos, 2, 0, gam, 1, 0, (int)n_rings, 2, 1, chordwise_only ? 1 : 0};
      UVLM_TRY(velocity_at(&v, 1, kNBodyFP64, dt, n_targets, vx, vy, vz, S));
    } else {
      UVLM_CUDA_TRY(cudaMemset(vx, 0, 8 * n_targets));
      UVLM_CUDA_TRY(cudaMemset(vy, 0, 8 * n_targets));
      UVLM_CUDA_TRY(cudaMemset(vz, 0, 8 * n_targets));
    }
    soa_to_aos<<<gfor(n_targets), 256>>>(vx, vy, vz, n_targets, dout, nullptr, nullptr, 1.0);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(out, dout, sizeof(double) * 3 * n_targets, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_rings_advect(const double* vortex_rings, const double* vortex_gamma, int64_t n_vortex, double* wake_rings,
                      int64_t n_wake, const double freestream[3], double dt) {
  if (n_vortex < 0 || n_wake < 0 || !freestream || (n_wake && !wake_rings) ||
      (n_vortex && (!vortex_rings || !vortex_gamma)))
    return report(fail(kErrInvalid, "invalid argument"));
  if (n_wake == 0) return UVLM_OK;
  Scratch S;
  auto run = [&]() -> Error {
    const long long nt = 4 * n_wake;
    double *dw, *vx, *vy, *vz, *dfs, *dr, *dg, *pos, *gam;
    UVLM_TRY(S.up(&dw, wake_rings, (size_t)(12 * n_wake)));
    UVLM_TRY(S.up(&dfs, freestream, 3));
    UVLM_TRY(S.get(&vx, nt));
    UVLM_TRY(S.get(&vy, nt));
    UVLM_TRY(S.get(&vz, nt));
    if (n_vortex > 0) {
      UVLM_TRY(S.up(&dr, vortex_rings, (size_t)(12 * n_vortex)));
      UVLM_TRY(S.up(&dg, vortex_gamma, (size_t)n_vortex));
      UVLM_TRY(S.get(&pos, 12 * n_vortex));
      UVLM_TRY(S.get(&gam, n_vortex));
      rings_to_sheets<<<gfor(n_vortex), 256>>>(dr, dg, n_vortex, pos, gam);
      UVLM_LAUNCH_CHECK();
      SheetView v{pos, 2, 0, gam, 1, 0, (int)n_vortex, 2, 1};
      UVLM_TRY(velocity_at(&v, 1, kNBodyFP64, dw, nt, vx, vy, vz, S));
    } else {
      UVLM_CUDA_TRY(cudaMemset(vx, 0, 8 * nt));
      UVLM_CUDA_TRY(cudaMemset(vy, 0, 8 * nt));
      UVLM_CUDA_TRY(cudaMemset(vz, 0, 8 * nt));
    }
    // node += (induced + freestream) * dt  (src/shed.inl:8-19)
    double* dout;
    UVLM_TRY(S.get(&dout, 3 * nt));
    soa_to_aos<<<gfor(nt), 256>>>(vx, vy, vz, nt, dout, dfs, dw, dt);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(wake_rings, dout, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_rings_connect_trailing_edge(const double* edge_rings, int64_t n_edge, double* wake_rings) {
  if (n_edge < 0 || (n_edge && (!edge_rings || !wake_rings))) return report(fail(kErrInvalid, "invalid argument"));
  if (n_edge == 0) return UVLM_OK;
  Scratch S;
  auto run = [&]() -> Error {
    double *de, *dw;
    UVLM_TRY(S.up(&de, edge_rings, (size_t)(12 * n_edge)));
    UVLM_TRY(S.up(&dw, wake_rings, (size_t)(12 * n_edge)));
    connect_te_kernel<<<gfor(n_edge), 256>>>(de, n_edge, dw);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(wake_rings, dw, sizeof(double) * 12 * n_edge, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_rings_solve_linear_problem(const double* bound_rings, const double* bound_rings0, int64_t n_bound,
                                    const double* wake_rings, const double* wake_gamma, int64_t n_wake,
                                    const double freestream[3], const uvlm_kinematics* kin, double t,
                                    int32_t drop_wake_term, double* gamma_out) {
  if (!bound_rings || n_bound < 1 || !freestream || !gamma_out || n_wake < 0 ||
      (n_wake && (!wake_rings || !wake_gamma)))
    return report(fail(kErrInvalid, "invalid argument"));
  uvlm_kinematics k{};
  if (kin) k = *kin;
  return report(solve_rings(bound_rings, bound_rings0, n_bound, &k, 1, nullptr, wake_rings, wake_gamma, n_wake,
                            freestream, t, drop_wake_term, gamma_out));
}

int uvlm_rings_solve_linear_problem_containers(const double* bound_rings, const double* bound_rings0,
                                               const int64_t* container_rings, int32_t n_containers,
                                               const uvlm_kinematics* kins, const double* wake_rings,
                                               const double* wake_gamma, int64_t n_wake,
                                               const double freestream[3], double t, int32_t drop_wake_term,
                                               double* gamma_out) {
  if (!bound_rings || n_containers < 1 || !container_rings || !kins || !freestream || !gamma_out || n_wake < 0 ||
      (n_wake && (!wake_rings || !wake_gamma)))
    return report(fail(kErrInvalid, "invalid argument"));
  std::vector<int> kin_of;
  for (int c = 0; c < n_containers; ++c) {
    if (container_rings[c] < 0) return report(fail(kErrInvalid, "negative container size"));
    kin_of.insert(kin_of.end(), (size_t)container_rings[c], c);
  }
  if (kin_of.empty()) return report(fail(kErrInvalid, "no bound rings"));
  return report(solve_rings(bound_rings, bound_rings0, (int64_t)kin_of.size(), kins, n_containers, kin_of.data(),
                            wake_rings, wake_gamma, n_wake, freestream, t, drop_wake_term, gamma_out));
}

int uvlm_lu_factor_f32(const float* A, int64_t n, int32_t update, float* LU, int32_t* ipiv) {
  if (!A || !LU || n < 1 || update < 0 || update > 2) return report(fail(kErrInvalid, "invalid argument"));
  if (update != 0 && !gemm_tc_available()) return report(fail(kErrUnsupported, "no tcgen05 device"));
  Scratch S;
  auto run = [&]() -> Error {
    const int N = (int)n;
    float* dA;
    UVLM_TRY(S.up(&dA, A, (size_t)N * N));
    LuWork lu;
    UVLM_TRY(lu_work_alloc(&lu, N, 4, sms()));
    const LuUpdate u = update == 0 ? kLuUpdateSimt : (update == 1 ? kLuUpdateTF32 : kLuUpdateBF16);
    Error e = lu_factor_f32(dA, N, u, &lu, 0);
    if (!e.code) e = lu_check(&lu, 0);
    if (!e.code && cudaMemcpy(LU, dA, sizeof(float) * (size_t)N * N, cudaMemcpyDeviceToHost) != cudaSuccess)
      e = fail(kErrCuda, "copy failed");
    if (!e.code && ipiv && cudaMemcpy(ipiv, lu.ipiv, sizeof(int) * N, cudaMemcpyDeviceToHost) != cudaSuccess)
      e = fail(kErrCuda, "copy failed");
    lu_work_free(&lu);
    return e;
  };
  return report(run());
}

int uvlm_dense_solve(const double* A, int64_t n, const double* b, double* x, int32_t method, int32_t* iters) {
  if (!A || !b || !x || n < 1 || method < 0 || method > 2) return report(fail(kErrInvalid, "invalid argument"));
  Scratch S;
  auto run = [&]() -> Error {
    const int N = (int)n;
    double *dA, *db, *dx, *tmp;
    UVLM_TRY(S.up(&dA, A, (size_t)N * N));
    UVLM_TRY(S.up(&db, b, (size_t)N));
    UVLM_TRY(S.get(&dx, (size_t)N));
    UVLM_TRY(S.get(&tmp, (size_t)N));
    LuWork lu;
    Error e;
    if (method == 0) {
      UVLM_TRY(lu_work_alloc(&lu, N, 8, sms()));
      e = lu_factor_f64(dA, N, &lu, 0);
      if (!e.code) e = lu_check(&lu, 0);
      if (!e.code) e = lu_solve_f64(dA, N, &lu, db, dx, tmp, 0);
      if (!e.code) e = lu_check(&lu, 0);
      if (iters) *iters = 0;
    } else {
      float* F;
      UVLM_TRY(S.get(&F, (size_t)N * N));
      f64_to_f32<<<gfor((long long)N * N), 256>>>(dA, (long long)N * N, F);
      UVLM_LAUNCH_CHECK();
      UVLM_TRY(lu_work_alloc(&lu, N, 4, sms()));
      const LuUpdate upd = method == 2 ? kLuUpdateBF16 : kLuUpdateTF32;
      e = lu_factor_f32(F, N, gemm_tc_available() ? upd : kLuUpdateSimt, &lu, 0);
      if (!e.code) e = lu_check(&lu, 0);
      GmresWork gw;
      GmresResult r;
      if (!e.code) e = gmres_work_alloc(&gw, N, 20);
      if (!e.code) {
        UVLM_CUDA_TRY(cudaMemset(dx, 0, sizeof(double) * N));
        e = gmres_solve(nullptr, dA, N, F, &lu, nullptr, db, dx, 1e-13, 200, &gw, &r, 0);
      }
      if (!e.code) e = lu_check(&lu, 0);
      gmres_work_free(&gw);
      if (!e.code && !r.converged) e = fail(kErrNonFinite, "GMRES did not converge");
      if (iters) *iters = r.iters;
    }
    lu_work_free(&lu);
    UVLM_TRY(e);
    UVLM_CUDA_TRY(cudaMemcpy(x, dx, sizeof(double) * N, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_rings_vortex_impulse(const double* rings, const double* gammas, int64_t n, double out[3]) {
  if (n < 0 || !out || (n && (!rings || !gammas))) return report(fail(kErrInvalid, "invalid argument"));
  Scratch S;
  auto run = [&]() -> Error {
    double *dr, *dg, *dout;
    UVLM_TRY(S.get(&dout, 3));
    if (n > 0) {
      UVLM_TRY(S.up(&dr, rings, (size_t)(12 * n)));
      UVLM_TRY(S.up(&dg, gammas, (size_t)n));
    } else {
      dr = dg = nullptr;
    }
    vortex_impulse_kernel<<<1, kSumThreads>>>(dr, dg, n, dout);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(out, dout, sizeof(double) * 3, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

int uvlm_rings_lamb_vector(const double* panels, const double* panel_gamma, const double* node_velocities,
                           int64_t n_panels, const double* freestreams, const double* vortices,
                           const double* vortex_gamma, int64_t n_vortices, double out[3]) {
  if (n_panels < 0 || n_vortices < 0 || !out ||
      (n_panels && (!panels || !panel_gamma || !node_velocities || !freestreams)) ||
      (n_vortices && (!vortices || !vortex_gamma)))
    return report(fail(kErrInvalid, "invalid argument"));
  Scratch S;
  auto run = [&]() -> Error {
    double *dp, *dg, *dv, *df, *dt, *vx, *vy, *vz, *du, *dout;
    UVLM_TRY(S.get(&dout, 3));
    const long long nt = 4 * n_panels;
    if (n_panels > 0) {
      UVLM_TRY(S.up(&dp, panels, (size_t)(12 * n_panels)));
      UVLM_TRY(S.up(&dg, panel_gamma, (size_t)n_panels));
      UVLM_TRY(S.up(&dv, node_velocities, (size_t)(12 * n_panels)));
      UVLM_TRY(S.up(&df, freestreams, (size_t)(3 * n_panels)));
      UVLM_TRY(S.get(&dt, 3 * nt));
      UVLM_TRY(S.get(&vx, nt));
      UVLM_TRY(S.get(&vy, nt));
      UVLM_TRY(S.get(&vz, nt));
      UVLM_TRY(S.get(&du, 3 * nt));
      lamb_midpoints_kernel<<<gfor(nt), 256>>>(dp, n_panels, dt);
      UVLM_LAUNCH_CHECK();
      if (n_vortices > 0) {
        // velocity of every vortex ring at the midpoints (InducedVelocityByVortices)
        double *dr, *drg, *pos, *gam;
        UVLM_TRY(S.up(&dr, vortices, (size_t)(12 * n_vortices)));
        UVLM_TRY(S.up(&drg, vortex_gamma, (size_t)n_vortices));
        UVLM_TRY(S.get(&pos, 12 * n_vortices));
        UVLM_TRY(S.get(&gam, n_vortices));
        rings_to_sheets<<<gfor(n_vortices), 256>>>(dr, drg, n_vortices, pos, gam);
        UVLM_LAUNCH_CHECK();
        SheetView v{pos, 2, 0, gam, 1, 0, (int)n_vortices, 2, 1, 0};
        UVLM_TRY(velocity_at(&v, 1, kNBodyFP64, dt, nt, vx, vy, vz, S));
      } else {
        UVLM_CUDA_TRY(cudaMemset(vx, 0, 8 * nt));
        UVLM_CUDA_TRY(cudaMemset(vy, 0, 8 * nt));
        UVLM_CUDA_TRY(cudaMemset(vz, 0, 8 * nt));
      }
      soa_to_aos<<<gfor(nt), 256>>>(vx, vy, vz, nt, du, nullptr, nullptr, 1.0);
      UVLM_LAUNCH_CHECK();
    } else {
      dp = dg = dv = df = du = nullptr;
    }
    lamb_sum_kernel<<<1, kSumThreads>>>(dp, dg, dv, df, n_panels, du, dout);
    UVLM_LAUNCH_CHECK();
    UVLM_CUDA_TRY(cudaMemcpy(out, dout, sizeof(double) * 3, cudaMemcpyDeviceToHost));
    return ok();
  };
  return report(run());
}

}  // extern "C"
