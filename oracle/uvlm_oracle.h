/*
 * uvlm_oracle.h -- C API of the CPU correctness oracle (TEST INFRASTRUCTURE).
 *
 * The oracle is a plain C++17, FP64, OpenMP restatement of xeno14/UVLM's
 * per-step time-stepper (SimpleSimulator) and of the legacy AoS vortex-ring
 * API.  It exists only to check the CUDA product and to serve as the timed
 * CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it; the product never does.
 *
 * Parity pin: the reference cannot be compiled here (Eigen3, protobuf, glog,
 * gflags, boost and the multiple_sheet submodule are absent), so the oracle is
 * pinned against the known-answer tests of the reference's own gtest suite
 * (test/vortex_test.cpp, test/shed_test.cpp, test/linear_test.cpp,
 * test/morphing_test.cpp, test/calc_load_test.cpp, test/wing_test.cpp,
 * test/rect_test.cpp), restated in tests/test_oracle_kats.py.
 *
 * Layout conventions (same as the product C-ABI):
 *  - A node sheet is MultipleSheet<Vector3d>(num, rows, cols) stored as
 *    contiguous [n][i][j][xyz] doubles (Vector3d is 3 packed doubles).
 *  - A circulation sheet is MultipleSheet<double>(num, rows, cols): [n][i][j].
 *  - An AoS ring is 4 nodes x 3 doubles (VortexRing::nodes()).
 */
#ifndef UVLM_ORACLE_H_
#define UVLM_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Closed-form kinematics (src/morphing.h:70-92 with the std::function
 * arguments replaced by sinusoid parameters); identical field layout to the
 * product's uvlm_kinematics.
 *   plug(t)     = plug_amp  * sin(plug_omega  * t + plug_phase)
 *   flap(t)     = flap_amp  * sin(flap_omega  * t + flap_phase)
 *   twist(x0,t) = (twist_amp + twist_span_slope*|y|) * sin(twist_omega*t + twist_phase)
 *   bend(x0,t)  = (bend_cx * x*(1-x) + bend_cy * y*y) * sin(bend_omega*t + bend_phase)
 * where (x, y) are the components of x_ref (mirrored to y >= 0). */
typedef struct {
  double alpha;
  double plug_amp, plug_omega, plug_phase;
  double flap_amp, flap_omega, flap_phase;
  double twist_amp, twist_span_slope, twist_omega, twist_phase;
  double bend_cx, bend_cy, bend_omega, bend_phase;
  double origin[3];
} orc_kinematics;

/* ---- L1 primitives: src/vortex.cpp, src/velocity.h ---------------------- */
void orc_biot_savart(const double start[3], const double end[3],
                     const double pos[3], double out[3]);
double orc_distance_line_and_point(const double start[3], const double end[3],
                                   const double pos[3]);
void orc_voring(const double* pos, int64_t pnum, int64_t prows, int64_t pcols,
                const double* gamma, int64_t grows, int64_t gcols, int64_t n,
                int64_t i, int64_t j, const double x[3], double out[3]);
void orc_sheet_induced_velocity(const double* pos, int64_t pnum, int64_t prows,
                                int64_t pcols, const double* gamma,
                                int64_t grows, int64_t gcols,
                                const double* targets, int64_t n_targets,
                                double* out);

/* ---- legacy AoS ring API: src/vortex.{h,cpp}, src/shed.inl -------------- */
void orc_ring_biot_savart(const double nodes[12], double gamma,
                          const double pos[3], double out[3]);
void orc_ring_chordwise_biot_savart(const double nodes[12], double gamma,
                                    const double pos[3], double out[3]);
/* what: 0 normal, 1 tangent, 2 tangent2, 3 centroid, 4 tanvec_chord,
 *       5 tanvec_span, 6 impulse (uses gamma) */
void orc_ring_vector(const double nodes[12], double gamma, int what,
                     double out[3]);
/* what: 0 area, 1 calc_c, 2 calc_b */
double orc_ring_scalar(const double nodes[12], int what);
double orc_ring_angle_of_attack(const double nodes[12], const double Q[3]);

/* ---- impulse post-processing: src/calc_impulse.h, calc_impulse_main.cpp -- */
/* Sum over rings of VortexRing::Impulse() (CalcVortexImpulse,
 * calc_impulse_main.cpp:34-41; vortex.cpp:140-143). */
void orc_vortex_impulse(const double* rings, const double* gammas, int64_t n, double out[3]);
/* Sum over panels of CalcLambVectorOnPanel(panel, v_nodes, freestream,
 * vortices) (calc_impulse.h:15-30); v_nodes: 4 x 3 per panel, one per
 * segment in ForEachSegment order; freestreams: 3 per panel. */
void orc_lamb_vector(const double* panels, const double* panel_gamma, const double* v_nodes, int64_t n_panels,
                     const double* freestreams, const double* vortices, const double* vortex_gamma,
                     int64_t n_vortices, double out[3]);
void orc_rings_induced_velocity(const double* rings, const double* gammas,
                                int64_t n_rings, const double pos[3],
                                int chordwise_only, double out[3]);
/* parallel=0: UVLM::Advect (serial, in-order); 1: UVLM::AdvectParallel */
void orc_rings_advect(const double* vortex_rings, const double* vortex_gamma,
                      int64_t n_vortex, double* wake_rings, int64_t n_wake,
                      const double freestream[3], double dt, int parallel);
void orc_connect_trailing_edge(const double* edge_rings, int64_t n_edge,
                               double* wake_rings);
/* UVLM::SolveLinearProblem (src/linear.inl:113-130).  drop_wake_term=1
 * reproduces the reference, whose wake RHS term is a discarded statement. */
int orc_solve_linear_problem(const double* bound_rings,
                             const double* bound_rings0, int64_t n_bound,
                             const double* wake_rings, const double* wake_gamma,
                             int64_t n_wake, const double freestream[3],
                             const orc_kinematics* m, double t,
                             int drop_wake_term, double* gamma_out);
/* SolveLinearProblem(containers, morphings, freestream, t) (src/linear.inl:
 * 132-157): container c has container_rings[c] bound rings and kins[c]. */
int orc_solve_linear_problem_containers(const double* bound_rings, const double* bound_rings0,
                                        const int64_t* container_rings, int n_containers,
                                        const orc_kinematics* kins, const double* wake_rings,
                                        const double* wake_gamma, int64_t n_wake, const double freestream[3],
                                        double t, int drop_wake_term, double* gamma_out);
/* calc_load::CalcLoadKatzPlotkin (src/calc_load/katz_plotkin.cpp:16-68);
 * out = F (3), Pin, Pout. */
void orc_load_katz_plotkin(const double* rings, const double* gamma, const double* gamma_prev, int64_t rows,
                           int64_t cols, const orc_kinematics* m, const double* bound_rings,
                           const double* bound_gamma, int64_t n_bound, const double* wake_rings,
                           const double* wake_gamma, int64_t n_wake, const double freestream[3], double rho,
                           double t, double dt, double out[5]);
/* container calc_load::CalcLoadJoukowski (src/calc_load/joukowski.h:24-104). */
void orc_load_joukowski_rings(const double* rings, const double* rings0, const double* gamma,
                              const double* gamma_prev, int64_t rows, int64_t cols, const orc_kinematics* m,
                              const double* vortices, const double* vortex_gamma, int64_t n_vortices,
                              const double freestream[3], double rho, double t, double dt, double out[5]);
void orc_calc_morphing_velocity_on_wing(const double* rings,
                                        const double* rings0, int64_t n,
                                        const orc_kinematics* m, double t,
                                        double* out);

/* ---- kinematics: src/morphing.cpp -------------------------------------- */
void orc_kin_perfome(const orc_kinematics* m, const double x0[3], double t,
                     double out[3]);
void orc_kin_velocity(const orc_kinematics* m, const double x0[3], double t,
                      double h, double out[3]);
void orc_calc_um(const orc_kinematics* m, const double x0[3],
                 const double freestream[3], double t, double out[3]);

/* ---- wing lattice: src/wing/rect.{h,cpp}, src/wing/wing.cpp ------------- */
void orc_transform_chebyshev(int64_t N, double xmin, double xmax, double* out);
/* RectGenerator(chord, half_span, rows, half_cols) -> (rows+1)*(half_cols+1)*3 */
void orc_rect_generate(double chord, double span, int64_t rows, int64_t cols,
                       int cheb_chord, int cheb_span, double* out);
/* WholeWing(half) with half origin: out is (rows+1)*(2*half_cols+1)*3 */
void orc_whole_wing(const double* half, int64_t rows, int64_t half_cols,
                    const double origin[3], double* out);

/* NACA4digit (src/wing/naca4digit.cpp:12-27) and NACA00XX
 * (src/wing/naca00XX.cpp:14-19) at x for chord c and digits xx. */
double orc_naca4digit(double x, double c, int xx);
double orc_naca00xx(double x, double c, int xx);
/* WingGenerator::Generate of RectGenerator (generator 0), NACA4digitGenerator
 * (1) or NACA00XXGenerator (2) with `digit`: (rows+1)*(cols+1)*3 points. */
void orc_generate_wing(int generator, int digit, double chord, double span, int64_t rows, int64_t cols, int cc,
                       int cs, double* out);

/* ---- dense solve: Eigen::FullPivLU<MatrixXd>(A).solve(b) ---------------- */
/* A is row-major n x n and is overwritten.  Returns 0, or 1 if singular. */
int orc_fullpiv_lu_solve(double* A, int64_t n, const double* b, double* x);

/* ---- SimpleSimulator (src/simulator/simple_simulator.{h,cpp}) ----------- */
void* orc_sim_create(void);
void orc_sim_destroy(void* sim);
int orc_sim_add_wing(void* sim, double chord, double span, int64_t rows,
                     int64_t cols, const double origin[3],
                     const orc_kinematics* m, int cheb_chord, int cheb_span);
/* AddWing with a NACA4digitGenerator (generator 1) or NACA00XXGenerator (2)
 * of the given digits; generator 0 is RectGenerator (= orc_sim_add_wing). */
int orc_sim_add_wing_generator(void* sim, int generator, int digit, double chord, double span, int64_t rows,
                               int64_t cols, const double origin[3], const orc_kinematics* m, int cheb_chord,
                               int cheb_span);
/* Threads of the FullPivLU elimination (default 1, as Eigen's).  The result
 * is bit-identical for any count. */
void orc_sim_set_lu_threads(void* sim, int threads);
void orc_sim_set_forward_flight(void* sim, const double ff[3]);
/* names as AdvectFactory: "euler", "RK2", "RK4", "AB2" */
int orc_sim_set_advection(void* sim, const char* name);
void orc_sim_set_erase_wake_after(void* sim, int64_t step);
void orc_sim_set_threads(void* sim, int threads);
/* Start of Run(): BuildWing + empty wake. */
int orc_sim_begin(void* sim);
/* One MainLoop(step, dt) and the optional erase; load_row gets
 * t, CD0, CL0, CD1, CL1, ... (1 + 2*num doubles) or NULL. */
int orc_sim_step(void* sim, int64_t step, double dt, double* load_row);
void orc_sim_sizes(void* sim, int64_t* num, int64_t* rows, int64_t* cols,
                   int64_t* wake_rows);
/* Node rows of wake_pos (wake_rows + 1 after the first step, 0 before). */
int64_t orc_sim_wake_node_rows(void* sim);
void orc_sim_get_state(void* sim, double* wing_pos, double* wing_pos_init,
                       double* wake_pos, double* wing_gamma,
                       double* wing_gamma_prev, double* wake_gamma);
/* Replace the state (positions and circulations) with a wake of wake_rows
 * ring rows (wake_rows + 1 node rows); the advection strategy is reset. */
int orc_sim_set_state(void* sim, int64_t wake_rows, const double* wing_pos,
                      const double* wake_pos, const double* wing_gamma,
                      const double* wing_gamma_prev, const double* wake_gamma);
/* MainLoop(step, dt) cut into `slices` consecutive slices of about equal
 * estimated time (threads: the OpenMP threads the N-body loops run with, used
 * for the estimate only).  Running every slice in order (orc_sim_sliced_run
 * with slice = 0, 1, ..., slices-1) performs exactly orc_sim_step(step, dt):
 * the same expressions for every output element.  load_row is written by the
 * slice that finishes the loads (pass it to every call).  Returns 0, 4 before
 * begin, 5 singular, 6 for a slice out of order. */
int orc_sim_sliced_begin(void* sim, int64_t step, double dt, int64_t slices, int threads);
int orc_sim_sliced_run(void* sim, int64_t slice, double* load_row);
/* Timing helper for the CPU baseline: runs every stage of MainLoop(step) on a
 * copy of the state, evaluating the N-body stages on every stride-th target
 * only and the FullPivLU on the leading lu_n x lu_n block.  Writes per-stage
 * seconds (kinematics+shed, assembly, rhs, solve, loads, advect) scaled to the
 * full stage (N-body by stride, LU by (N/lu_n)^3).  State is not modified. */
int orc_sim_time_step_sampled(void* sim, int64_t step, double dt,
                              int64_t stride, int64_t lu_n,
                              double* stage_seconds);

#ifdef __cplusplus
}
#endif
#endif  // UVLM_ORACLE_H_
