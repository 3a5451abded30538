// step.cuh -- per-step kernels of the time-stepper other than the N-body and
// the dense solve: kinematics, shedding, panel geometry, influence-matrix
// assembly, RHS, Joukowski loads and the advection updates.
#pragma once

#include "../../include/uvlm_b200.h"
#include "common.cuh"

namespace uvlm {

// Physical layout of a wake sheet set: node row i (logical, 0 = newest, the
// trailing edge) of sheet n lives at physical row start + i of a buffer of
// PR rows per sheet; ring row i shares physical row start + i.  Shedding
// writes row start-1 and decrements start (an O(C) prepend).
struct WakeLayout {
  int num, C, PR, start, node_rows;
  __host__ __device__ long long node(int n, int i, int j) const {
    return ((long long)n * PR + start + i) * (C + 1) + j;
  }
  __host__ __device__ long long ring(int n, int i, int j) const {
    return ((long long)n * PR + start + i) * C + j;
  }
};

struct WingShape {
  int num, R, C;  // rings per wing R x C
  __host__ __device__ long long node(int n, int i, int j) const { return ((long long)n * (R + 1) + i) * (C + 1) + j; }
  __host__ __device__ long long ring(int n, int i, int j) const { return ((long long)n * R + i) * C + j; }
  __host__ __device__ int lines_per_wing() const { return R * (2 * C + 1); }
};

Error launch_kinematics(const uvlm_kinematics* d_kin, WingShape ws, const double* pos_init, double* pos, double t,
                        cudaStream_t st);
Error launch_shed(WingShape ws, const double* wing_pos, const double* wing_gamma, WakeLayout wl, double* wake_pos,
                  double* wake_gamma, bool shed_gamma, cudaStream_t st);
// collocation points (SoA), normals, panel areas, morphing velocity at the
// reference collocation points (simple_simulator.cpp:19-50, :103-124).
Error launch_panel_geometry(const uvlm_kinematics* d_kin, WingShape ws, const double* pos, const double* pos_init,
                            double t, double* cx, double* cy, double* cz, double* normal, double* area, double* uls,
                            cudaStream_t st);
// A[K][L] = VORING(c_K, L, Gamma=1) . n_K (simple_simulator.cpp:76-101),
// FP64 or FP32-hi/lo arithmetic, row-major output of type float or double.
Error launch_assemble(WingShape ws, const double* pos, const double* cx, const double* cy, const double* cz,
                      const double* normal, bool fp32, void* A, bool out_f32, cudaStream_t st);
// AoS-ring assembly of the legacy SolveLinearProblem (src/linear.inl:14-32).
Error launch_assemble_rings(const double* rings, int n, double* A, double* centroid, double* normal,
                            cudaStream_t st);
// Legacy RHS (src/linear.inl:34-76, :113-130): b_i = Vls(ref centroid_i).n_i
// - freestream.n_i [- wake(centroid_i).n_i when the wake term is kept].
// Ring i moves with d_kin[d_kin_of[i]] (d_kin_of NULL: d_kin[0]), the
// per-container morphings of CalcRhsMorphings (src/linear.inl:87-104).
Error launch_legacy_rhs(const uvlm_kinematics* d_kin, const int* d_kin_of, const double* rings0, int n,
                        const double* centroid, const double* normal, const double fs[3], double t,
                        const double* wake_vel, double* b, cudaStream_t st);
// b_K = -(Uw - (Uls + ff)) . n_K
Error launch_rhs(int N, const double* uw_x, const double* uw_y, const double* uw_z, const double* uls,
                 const double* normal, const double ff[3], double* b, cudaStream_t st);
// unique load lines: midpoints (targets) and morphing velocity at the
// reference midpoints (joukowski.cpp:12-34 + simple_simulator.cpp:203-211).
Error launch_line_prep(const uvlm_kinematics* d_kin, WingShape ws, const double* pos, const double* pos_init,
                       double t, double* tx, double* ty, double* tz, double* line_uls, cudaStream_t st);
// Joukowski steady + unsteady force and coefficients per wing into row.
Error launch_loads(WingShape ws, const double* pos, const double* gamma, const double* gamma_prev,
                   const double* normal, const double* area, const double* vx, const double* vy, const double* vz,
                   const double* line_uls, const double ff[3], const double* chord_span, double t, double dt,
                   double* row, cudaStream_t st);
// wake node rows first_row..node_rows-1 of pos into SoA targets (row 0, the
// trailing edge, moves with -ff alone)
Error launch_gather_wake(WakeLayout wl, const double* pos, double* tx, double* ty, double* tz, cudaStream_t st,
                         int first_row = 1);

enum AdvectMode {
  kAdvEuler = 0,
  kAdvRK2K1 = 1,    // k1 = u; pos2 = x + k1 dt
  kAdvRK2Upd = 2,   // k2 = u; x = x + (k1+k2) dt/2 (rows > ignore) else x + k1 dt
  kAdvRK4K1 = 3,    // k1 = u; pos2 = x + k1 dt/2
  kAdvRK4K2 = 4,    // k2 = u; pos2 = x + k2 dt/2
  kAdvRK4Upd = 5,   // k3 = u; x = x + (k1 + 2k2 + 2k3 + k3) dt/6 (rows > ignore) else x + k1 dt
  kAdvAB2 = 6,      // v = u; x = x + (3v - v_prev) dt/2 (rows >= 1, with history) else x + v dt
};
// u = -ff + vel (rows >= vrow0, vel indexed like launch_gather_wake with
// first_row = vrow0) or -ff (rows above vrow0; for kAdvRK2Upd and kAdvRK4Upd
// with vrow0 = ignore_rows + 1 those rows take the Euler step and do not read u)
Error launch_advect(AdvectMode mode, WakeLayout wl, double* x, double* pos2, double* k1, double* k2, double* k3,
                    double* vprev, bool has_vprev, const double* vx, const double* vy, const double* vz,
                    const double ff[3], double dt, int ignore_rows, cudaStream_t st, int vrow0 = 1);
// in-place relocation of the live wake rows (compaction of the prepend buffer)
Error launch_move_rows(double* buf, int num, int PR, int row_elems, int from, int to, int rows, double* tmp,
                       cudaStream_t st);
// x = 2 a - b (linear extrapolation of the circulation history)
Error launch_extrapolate(double* x, const double* a, const double* b, int n, cudaStream_t st);
// flag[0] |= any non-finite value in x[0..n)
Error launch_check_finite(const double* x, long long n, int* flag, cudaStream_t st);

}  // namespace uvlm
