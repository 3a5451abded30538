/*
 * uvlm_b200.h -- C-ABI of the B200 (sm_100a) UVLM time-stepper.
 *
 * Drop-in boundary for the per-step hot path of xeno14/UVLM: plain pointers
 * and sizes, no C++ or torch types.  Host arrays are borrowed only for the
 * duration of a call (copied in or out); all simulation state lives in HBM
 * inside an opaque context.  Every function returns a status code (0 = OK);
 * uvlm_last_error() gives the message of the last failure on a context, and
 * uvlm_global_last_error() that of the context-free entry points.
 *
 * Layouts (the reference's MultipleSheet, whose element K sits at
 * j + cols*(i + rows*n), with Eigen::Vector3d = 3 packed doubles):
 *   node sheet  (num, rows+1, cols+1) x 3 doubles  [n][i][j][xyz]
 *   gamma sheet (num, rows,   cols)       doubles  [n][i][j]
 *   AoS ring    4 nodes x 3 doubles (VortexRing::nodes())
 *
 * Reference interfaces replaced (paths inside xeno14/UVLM):
 *   SimpleSimulator::{AddWing,Run,MainLoop,set_forward_flight,set_advection}
 *       src/simulator/simple_simulator.h:50-63, simple_simulator.cpp:126-313
 *   advect::Advection::Advect + AdvectFactory
 *       src/advect.h:48-59, src/advect_factory.cpp:43-60
 *   UVLM::InducedVelocity(x, pos, gamma)          src/velocity.h:14-24
 *   UVLM::InducedVelocity / ChordwiseInducedVelocity / Advect /
 *       AdvectParallel / ConnectTrailingEdge (AoS) src/shed.h:14-46
 *   UVLM::SolveLinearProblem (AoS)                src/linear.h:104-119
 *   Eigen::FullPivLU<MatrixXd>(A).solve(b)        src/simulator/simple_simulator.cpp:264-268
 */
#ifndef UVLM_B200_H_
#define UVLM_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define UVLM_OK 0
#define UVLM_ERR_INVALID 1     /* bad argument, shape or name */
#define UVLM_ERR_CUDA 2        /* CUDA runtime error */
#define UVLM_ERR_SINGULAR 3    /* zero pivot in the LU factorisation */
#define UVLM_ERR_NONFINITE 4   /* non-finite circulation after the solve */
#define UVLM_ERR_STATE 5       /* call out of order (e.g. step before begin) */
#define UVLM_ERR_CAPACITY 6    /* wake longer than max_wake_rows */
#define UVLM_ERR_TIMEOUT 7     /* a bounded device-side wait gave up */
#define UVLM_ERR_UNSUPPORTED 8 /* size or option outside what is built */

/* Advection schemes: AdvectFactory names "euler", "RK2", "RK4", "AB2". */
#define UVLM_ADVECT_EULER 0
#define UVLM_ADVECT_RK2 1
#define UVLM_ADVECT_RK4 2
#define UVLM_ADVECT_AB2 3

/* Arithmetic of the N-body, assembly and factorisation stages. */
#define UVLM_PRECISION_FP64 0  /* plain form: FP64 everywhere, fresh LU each step */
#define UVLM_PRECISION_MIXED 1 /* FP32 N-body/assembly, TF32/BF16 LU, FP64 residual */

/* Dense solve strategy. */
#define UVLM_SOLVER_LU 0          /* factor + solve every step (the reference's method) */
#define UVLM_SOLVER_GMRES_STALE 1 /* GMRES, FP64 residual, preconditioned by stale LU */

/* Initial guess of the GMRES solve. */
#define UVLM_WARM_PREVIOUS 0    /* previous step's circulation */
#define UVLM_WARM_EXTRAPOLATE 1 /* 2*Gamma_n - Gamma_{n-1} */
#define UVLM_WARM_MLP 2         /* learned warm start (uvlm_set_mlp) */

/* How the stale FP32 factors precondition the GMRES solve. */
#define UVLM_PRECOND_INVERSE 0    /* dense FP32 (LU)^-1 P formed once per factorisation; one matvec per iteration */
#define UVLM_PRECOND_TRIANGULAR 1 /* forward + backward triangular solves with the factors every iteration */

/* Factor precision of the mixed form (trailing updates on tcgen05). */
#define UVLM_LU_TF32 0
#define UVLM_LU_BF16 1

typedef struct uvlm_ctx uvlm_ctx;

typedef struct {
  int32_t precision;        /* UVLM_PRECISION_* */
  int32_t solver;           /* UVLM_SOLVER_* */
  int32_t warm_start;       /* UVLM_WARM_* */
  int32_t lu_precision;     /* UVLM_LU_* (mixed form) */
  int32_t advection;        /* UVLM_ADVECT_* */
  int32_t rk_ignore_rows;   /* RK2/RK4 use Euler for wake rows i <= this (5, src/advect.h:77) */
  int64_t max_wake_rows;    /* capacity in ring rows */
  int64_t erase_wake_after; /* --erase_wake_after (0 = never) */
  int32_t gmres_restart;    /* Krylov dimension before a restart */
  int32_t gmres_max_iter;   /* above this the plain fresh FP64 LU solve is taken (the fallback), and
                               the FP32 factors of the preconditioner are refreshed */
  double gmres_tol;         /* relative residual ||b - A g|| / ||b|| */
  int32_t device;           /* CUDA device ordinal */
  int32_t compute_loads;    /* 1: Joukowski loads every step (CalcLoad) */
  int32_t assembly_fp64;    /* mixed form: residual matrix assembled in FP64 each step
                               (the FP32 kernel then assembles only the matrix that is
                               factored); 0: FP32 assembly serves both */
  int32_t nbody_variant;    /* -1: autotune; else a tile variant index */
  int32_t preconditioner;   /* UVLM_PRECOND_* (mixed form, GMRES solver) */
  int32_t nbody_fp64_stages; /* mixed form: N-body stages evaluated in FP64 instead of FP32,
                                a mask of UVLM_STAGE_RHS | UVLM_STAGE_LOADS | UVLM_STAGE_ADVECT
                                (0: all FP32) */
  int32_t nbody_near_fp64;   /* mixed form: FP32 N-body stages (a mask of UVLM_STAGE_*) whose pairs the
                                far-field test leaves to the near-field walker (source strips close to
                                the targets) are evaluated in FP64 from FP64 records and accumulated in
                                FP64; 0: none; uvlm_config_default sets UVLM_STAGE_RHS */
  int32_t lu_pivoting;       /* mixed form, the factors of the GMRES preconditioner: UVLM_PIVOT_PANEL
                                (pivots chosen over every row of a 64-column panel) or UVLM_PIVOT_LOCAL
                                (over the panel's top 256 rows only, the default: a cheaper panel for
                                diagonally heavy influence matrices; GMRES with FP64 residuals and the
                                plain fresh-LU fallback keep the answer whatever the pivots) */
  int32_t gmres_refresh_iter; /* mixed form, GMRES solver: a step whose GMRES took at least this many
                                 iterations has the preconditioner refactored from the next step's
                                 matrix (0: only when gmres_max_iter is exceeded, the fallback); the
                                 default 16 refreshes aging factors before they reach the fallback */
} uvlm_config;

#define UVLM_PIVOT_PANEL 0
#define UVLM_PIVOT_LOCAL 1

/* N-body stages of a MainLoop (uvlm_config.nbody_fp64_stages). */
#define UVLM_STAGE_RHS 1    /* wake normal wash at the collocation points (CalcRhs) */
#define UVLM_STAGE_LOADS 2  /* velocities at the load-line midpoints (CalcLoad) */
#define UVLM_STAGE_ADVECT 4 /* velocities at the wake nodes (Advect) */

/* Closed-form kinematics of one wing (Morphing, src/morphing.h:70-92, with the
 * std::function arguments replaced by sinusoids):
 *   plug(t)     = plug_amp * sin(plug_omega * t + plug_phase)
 *   flap(t)     = flap_amp * sin(flap_omega * t + flap_phase)
 *   twist(x0,t) = (twist_amp + twist_span_slope*|y|) * sin(twist_omega*t + twist_phase)
 *   bend(x0,t)  = (bend_cx*x*(1-x) + bend_cy*y*y) * sin(bend_omega*t + bend_phase)
 * with (x, y) taken from x_ref = x0 - origin mirrored to y >= 0.  The velocity
 * is the reference's FP64 central difference with h = 1e-6. */
typedef struct {
  double alpha;
  double plug_amp, plug_omega, plug_phase;
  double flap_amp, flap_omega, flap_phase;
  double twist_amp, twist_span_slope, twist_omega, twist_phase;
  double bend_cx, bend_cy, bend_omega, bend_phase;
  double origin[3];
} uvlm_kinematics;

/* One rectangular wing: RectGenerator + WholeWing of AddWing/BuildWing
 * (src/simulator/simple_simulator.cpp:126-169, src/wing/rect.cpp:18-45,
 * src/wing/wing.cpp:12-52).  cols must be even. */
typedef struct {
  double chord, span;
  int64_t rows, cols;
  double origin[3];
  int32_t chebyshev_chord, chebyshev_span;
} uvlm_wing_desc;

typedef struct {
  int64_t step;
  double t;
  int32_t solve_path;   /* 0 fresh LU, 1 GMRES with stale LU, 2 the fallback: GMRES stopped at
                           gmres_max_iter (or its initial guess was non-finite) and the plain
                           fresh FP64 LU solve of the step's FP64 matrix gave the circulation */
  int32_t gmres_iters;
  double residual;      /* final ||b - A g|| / ||b|| (FP64), 0 for the plain LU path */
  int32_t refactored;   /* a factorisation ran in this step */
  int32_t wake_rows;    /* ring rows of the wake after the step */
  double stage_ms[8];   /* kinematics+shed, assembly, rhs, solve, loads, advect, warm start, total */
  int32_t nbody_variant; /* N-body tile variant in use (see uvlm_nbody_variant_name) */
  int32_t pad_;
  double initial_residual; /* ||b - A g0|| / ||b|| of the GMRES initial guess */
  double nbody_ms;         /* with stage timing: device time of the step's N-body launches */
  double factor_ms;        /* with stage timing, mixed form: device time of this step's FP32 LU (0 if none) */
  double inverse_ms;       /* ... and of the dense inverse of its factors (0 if none) */
  int32_t stage_variant[4]; /* N-body tile of the rhs, loads and advect stages ([3] = -1); nbody_variant
                               is the advect stage's in the context's precision */
} uvlm_step_stats;

/* ------------------------------------------------------- time-stepper */
void uvlm_config_default(uvlm_config* cfg);
int uvlm_create(const uvlm_config* cfg, uvlm_ctx** out);
int uvlm_destroy(uvlm_ctx* ctx);
const char* uvlm_last_error(const uvlm_ctx* ctx);
const char* uvlm_global_last_error(void);
const char* uvlm_status_string(int status);

/* SimpleSimulator::AddWing (simple_simulator.cpp:126-140): all wings must
 * share rows and cols, cols even. */
int uvlm_add_wing(uvlm_ctx* ctx, const uvlm_wing_desc* wing, const uvlm_kinematics* kin);
/* SimpleSimulator::AddWing with any wing::WingGenerator
 * (simple_simulator.h:50-53, simple_simulator.cpp:126-169): nodes is the
 * whole-wing lattice the generator and WholeWing produce ((rows + 1) x
 * (cols + 1) points of 3 doubles, [i][j][xyz], relative to the wing origin;
 * e.g. the NACA 4-digit camber lattice of src/wing/naca4digit.cpp:29-39).
 * The context adds `origin` to every node and sets the morphing origin to
 * it, as BuildWing does.  chord and span scale the load coefficients
 * (CalcLoad :227-229).  All wings share rows and cols. */
int uvlm_add_wing_nodes(uvlm_ctx* ctx, int64_t rows, int64_t cols, const double* nodes, double chord, double span,
                        const double origin[3], const uvlm_kinematics* kin);
/* SimpleSimulator::set_forward_flight (simple_simulator.h:57). */
int uvlm_set_forward_flight(uvlm_ctx* ctx, const double ff[3]);
/* SimpleSimulator::set_advection + AdvectFactory(name). */
int uvlm_set_advection(uvlm_ctx* ctx, const char* name);
/* Prologue of SimpleSimulator::Run (simple_simulator.cpp:288-303): builds
 * the wings and an empty wake; resets AB2 history. */
int uvlm_begin(uvlm_ctx* ctx);
/* SimpleSimulator::MainLoop(step, dt) plus the optional erase
 * (simple_simulator.cpp:240-286, 307-311).  load_row (host, may be NULL)
 * receives t, CD0, CL0, CD1, CL1, ... (1 + 2*num doubles, CalcLoad :226-232). */
int uvlm_step(uvlm_ctx* ctx, int64_t step, double dt, double* load_row);
/* The same MainLoop one stage at a time, for callers that act between the
 * stages (read the circulations before the loads, time a stage, ...).
 * uvlm_step is exactly these six calls, in this order; each call returns
 * UVLM_ERR_STATE when it is not the stage expected next, and an error in a
 * stage abandons the step (the next call must be uvlm_stage_kinematics).
 * uvlm_step, uvlm_set_state and uvlm_erase_oldest_wake are refused while a
 * staged step is in progress; uvlm_get_state may be called between stages.
 *   kinematics  Morphing of every wing, Shed(step), collocation points and
 *               normals (simple_simulator.cpp:241-262)
 *   assemble    CalcMatrix (:76-101)
 *   rhs         CalcRhs (:103-124)
 *   solve       the circulation solve (:264-268) and the per-step state
 *               output (:270-277)
 *   loads       CalcLoad (:195-233), when loads are computed
 *   advect      Advect(dt) (:284), the optional erase (:307-311), and the
 *               load row (as uvlm_step's) */
int uvlm_stage_kinematics(uvlm_ctx* ctx, int64_t step, double dt);
int uvlm_stage_assemble(uvlm_ctx* ctx);
int uvlm_stage_rhs(uvlm_ctx* ctx);
int uvlm_stage_solve(uvlm_ctx* ctx);
int uvlm_stage_loads(uvlm_ctx* ctx);
int uvlm_stage_advect(uvlm_ctx* ctx, double* load_row);
/* SimpleSimulator::Run(steps, dt): begin + steps+1 MainLoops; loads (host,
 * may be NULL) receives (steps+1) rows of 1 + 2*num doubles. */
int uvlm_run(uvlm_ctx* ctx, int64_t steps, double dt, double* loads);
/* SimpleSimulator::EraseOldestWake (simple_simulator.cpp:235-238). */
int uvlm_erase_oldest_wake(uvlm_ctx* ctx);
int uvlm_get_sizes(const uvlm_ctx* ctx, int64_t* num, int64_t* rows, int64_t* cols, int64_t* wake_rows,
                   int64_t* wake_node_rows);
/* Copies of the state (host arrays in the MultipleSheet layouts above; any
 * pointer may be NULL).  wake_pos has wake_node_rows rows. */
int uvlm_get_state(uvlm_ctx* ctx, double* wing_pos, double* wing_pos_init, double* wake_pos, double* wing_gamma,
                   double* wing_gamma_prev, double* wake_gamma);
/* Replaces positions and circulations with a wake of wake_rows ring rows
 * (wake_rows + 1 node rows); clears AB2 history and the stale factors. */
int uvlm_set_state(uvlm_ctx* ctx, int64_t wake_rows, const double* wing_pos, const double* wake_pos,
                   const double* wing_gamma, const double* wing_gamma_prev, const double* wake_gamma);
int uvlm_get_last_stats(const uvlm_ctx* ctx, uvlm_step_stats* stats);
/* 1: record per-stage times with CUDA events (adds synchronisation). */
int uvlm_set_stage_timing(uvlm_ctx* ctx, int32_t enable);
int uvlm_synchronize(uvlm_ctx* ctx);
/* The CUDA stream the context launches on (cudaStream_t), for callers that
 * time or order work around uvlm_step. */
void* uvlm_stream(uvlm_ctx* ctx);
/* Number of CUDA kernels this library has launched in this process (all
 * contexts and entry points); differences bracket a region of interest. */
int64_t uvlm_kernel_launch_count(void);
/* Measured FP32 FMA throughput of the device (TFLOP/s, the larger of a
 * scalar FFMA and a packed FP32x2 probe): the denominator of the FP32
 * N-body roofline.  No counterpart in the reference (measurement aid). */
int uvlm_measure_fp32_peak(int32_t device, double* tflops);
/* Measured FP64 FMA throughput (TFLOP/s): the denominator of the plain FP64
 * form's N-body roofline. */
int uvlm_measure_fp64_peak(int32_t device, double* tflops);
/* Every bounded device-side wait of the library (the triangular solves'
 * block-row flags, the cooperative grid barrier, the tensor-core kernels'
 * mbarriers) gives up after `cycles` SM clock cycles on `device` (0 restores
 * the default, about one second), flags the error word and returns; the call
 * that launched it returns UVLM_ERR_TIMEOUT.  No counterpart in the reference;
 * a knob for tests of the timeout path. */
int uvlm_set_wait_limit(int32_t device, int64_t cycles);
/* Check of the timeout path: one CTA waits (as a triangular-solve block row
 * waits for the rows before it) for a flag that nothing sets, with a limit of
 * `cycles`; the wait gives up and this returns UVLM_ERR_TIMEOUT.  The default
 * limit is restored afterwards and the device stays usable.  No counterpart
 * in the reference. */
int uvlm_check_bounded_wait(int32_t device, int64_t cycles);
/* Name of an N-body tile variant (e.g. "fp32_h4_t2_b128"), "?" if out of range. */
const char* uvlm_nbody_variant_name(int32_t variant);
/* Algorithmic work of the last step: unique-segment interactions of every
 * N-body stage and the assembly (target x segment pairs). */
int uvlm_get_last_work(const uvlm_ctx* ctx, double* nbody_pairs, double* assembly_pairs, double* lu_flops);

/* SimpleSimulator::Velocity (simple_simulator.h:98-100) at n arbitrary points
 * (targets, out: n x 3 host arrays): the bound and wake sheets' induced
 * velocity of the current state, minus the forward flight when
 * include_freestream != 0 (the reference's velocity-field tools, e.g.
 * src/tools/3d_velocity_main.cpp:73-78, evaluate this on grids). */
int uvlm_velocity_at(uvlm_ctx* ctx, const double* targets, int64_t n, int32_t include_freestream, double* out);

/* ------------------------------------------- context-free reference API */
/* UVLM::InducedVelocity(x, pos, gamma) for n_targets points
 * (src/velocity.h:14-24).  pos: (num, grows+1, gcols+1) nodes; gamma:
 * (num, grows, gcols); targets/out: n_targets x 3.  precision: UVLM_PRECISION_*. */
int uvlm_sheet_induced_velocity(const double* pos, const double* gamma, int64_t num, int64_t grows, int64_t gcols,
                                const double* targets, int64_t n_targets, double* out, int32_t precision);

/* No counterpart in the reference.  The same velocities as
 * uvlm_sheet_induced_velocity for callers that cannot allocate device memory
 * (loops where cudaMalloc/cudaFree would synchronise the device, or a host
 * framework that owns the device memory budget).  pos, gamma, targets and out
 * are DEVICE pointers owned by the caller; nothing is allocated.  An empty
 * sheet set (num, grows or gcols 0; pos and gamma may then be NULL) gives
 * zero velocities.  All scratch lives in one 32 MiB device array inside the
 * library (held by every GPU that loads it until exit); a request that needs
 * more returns UVLM_ERR_CAPACITY.  The first call on a device looks up that
 * array's address, so make it before any stream capture.  Work is queued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and is not
 * synchronised.  Calls share the array: calls that overlap on the GPU race. */
int uvlm_sheet_induced_velocity_noalloc(const double* pos, const double* gamma, int64_t num, int64_t grows,
                                        int64_t gcols, const double* targets, int64_t n_targets, double* out,
                                        int32_t precision, void* stream);

/* advect::Advection strategy object (src/advect.h:48-59) from
 * AdvectFactory(name) (src/advect_factory.cpp:43-60): "euler", "RK2",
 * "RK4", "AB2".  AB2 keeps its velocity history between calls. */
typedef struct uvlm_advection uvlm_advection;
int uvlm_advection_create(const char* name, int32_t precision, uvlm_advection** out);
int uvlm_advection_destroy(uvlm_advection* adv);
/* Advection::Advect(next, wing_pos, wing_gamma, wake_pos, wake_gamma,
 * forward_flight, dt).  Shapes: wing (num, rows, cols) rings, wake
 * (num, wake_rows, cols) rings with wake_rows + 1 node rows.  `next` may alias
 * `wake_pos` (simple_simulator.cpp:190-193). */
int uvlm_advection_advect(uvlm_advection* adv, double* next, const double* wing_pos, const double* wing_gamma,
                          int64_t num, int64_t rows, int64_t cols, const double* wake_pos, const double* wake_gamma,
                          int64_t wake_rows, const double forward_flight[3], double dt);

/* UVLM::InducedVelocity / ChordwiseInducedVelocity over AoS rings
 * (src/shed.inl:22-33, 66-77) for n_targets points. */
int uvlm_rings_induced_velocity(const double* rings, const double* gammas, int64_t n_rings, const double* targets,
                                int64_t n_targets, int32_t chordwise_only, double* out);
/* UVLM::AdvectParallel (src/shed.inl:52-64): every node of every wake ring
 * moves by (induced + freestream) * dt, velocities taken before any move. */
int uvlm_rings_advect(const double* vortex_rings, const double* vortex_gamma, int64_t n_vortex, double* wake_rings,
                      int64_t n_wake, const double freestream[3], double dt);
/* UVLM::ConnectTrailingEdge (src/shed.inl:79-86). */
int uvlm_rings_connect_trailing_edge(const double* edge_rings, int64_t n_edge, double* wake_rings);
/* UVLM::SolveLinearProblem (src/linear.inl:113-130).  drop_wake_term = 1
 * reproduces the reference, whose wake RHS term is a discarded statement
 * (src/linear.inl:123-124); 0 subtracts the wake normal wash. */
int uvlm_rings_solve_linear_problem(const double* bound_rings, const double* bound_rings0, int64_t n_bound,
                                    const double* wake_rings, const double* wake_gamma, int64_t n_wake,
                                    const double freestream[3], const uvlm_kinematics* kin, double t,
                                    int32_t drop_wake_term, double* gamma_out);
/* UVLM::SolveLinearProblem(containers, morphings, freestream, t)
 * (src/linear.inl:132-157): the bound rings of n_containers containers laid
 * out one after another (container c has container_rings[c] rings and moves
 * with kins[c], CalcRhsMorphings :87-104), then the wake rings.  FP64
 * assembly and LU; drop_wake_term as in uvlm_rings_solve_linear_problem. */
int uvlm_rings_solve_linear_problem_containers(const double* bound_rings, const double* bound_rings0,
                                               const int64_t* container_rings, int32_t n_containers,
                                               const uvlm_kinematics* kins, const double* wake_rings,
                                               const double* wake_gamma, int64_t n_wake,
                                               const double freestream[3], double t, int32_t drop_wake_term,
                                               double* gamma_out);
/* Morphing::Perfome / Morphing::Velocity (src/morphing.cpp:23-52) of n
 * reference points x0 [n][3] at time t. */
int uvlm_kinematics_perfome(const uvlm_kinematics* kin, const double* x0, int64_t n, double t, double* out);
int uvlm_kinematics_velocity(const uvlm_kinematics* kin, const double* x0, int64_t n, double t, double* out);
/* calc_load::CalcLoadKatzPlotkin(c, cp, morphing, rings, freestream, rho, t,
 * dt) (src/calc_load/katz_plotkin.cpp:16-68) for one container of rows x
 * cols rings (gamma: c, gamma_prev: cp).  The UVLMVortexRing `rings` is
 * given as its bound rings (chordwise velocity, uvlm_vortex_ring.h:80-83)
 * and wake rings (:75-78); n = 0 for the empty one the legacy simulator
 * passes (src/simulator/simulator.cpp:37,183).  out = F.x, F.y, F.z, Pin,
 * Pout; F starts from zero (the reference leaves it uninitialised) and Pout
 * is 0 as in the reference. */
int uvlm_rings_load_katz_plotkin(const double* rings, const double* gamma, const double* gamma_prev, int64_t rows,
                                 int64_t cols, const uvlm_kinematics* kin, const double* bound_rings,
                                 const double* bound_gamma, int64_t n_bound, const double* wake_rings,
                                 const double* wake_gamma, int64_t n_wake, const double freestream[3], double rho,
                                 double t, double dt, double out[5]);
/* calc_load::CalcLoadJoukowski(vb, vb_prev, morphing, freestream, rho, t, dt)
 * (src/calc_load/joukowski.h:24-104) for one container: rings / rings0 are
 * its nodes() / nodes0(); the induced velocity at the segment midpoints
 * comes from every ring of `vortices` (the container's whole ring pool).
 * out = F.x, F.y, F.z, Pin, Pout = -F.x |freestream|. */
int uvlm_rings_load_joukowski(const double* rings, const double* rings0, const double* gamma,
                              const double* gamma_prev, int64_t rows, int64_t cols, const uvlm_kinematics* kin,
                              const double* vortices, const double* vortex_gamma, int64_t n_vortices,
                              const double freestream[3], double rho, double t, double dt, double out[5]);
/* Impulse post-processing (src/calc_impulse_main.cpp:51-83), FP64.
 * Sum over rings of VortexRing::Impulse() = -Normal * gamma * Area
 * (CalcVortexImpulse, calc_impulse_main.cpp:34-41; vortex.cpp:140-143). */
int uvlm_rings_vortex_impulse(const double* rings, const double* gammas, int64_t n, double out[3]);
/* Sum over panels of calc_impulse::CalcLambVectorOnPanel(panel_i,
 * node_velocities_i, freestreams_i, vortices) (calc_impulse.h:15-30, summed
 * as calc_impulse_main.cpp:79-82): node_velocities [n_panels][4][3], one per
 * segment in ForEachSegment order; freestreams [n_panels][3]; the induced
 * velocity at each segment midpoint comes from every ring of `vortices`. */
int uvlm_rings_lamb_vector(const double* panels, const double* panel_gamma, const double* node_velocities,
                           int64_t n_panels, const double* freestreams, const double* vortices,
                           const double* vortex_gamma, int64_t n_vortices, double out[3]);
/* ------------------------------------------------- per-step state output */
/* SimpleSimulator::set_sheet_path / set_result_path
 * (src/simulator/simple_simulator.cpp:53-66): from the next step on, every
 * MainLoop writes the state after its solve as one AllVortexSheets record
 * (OutputSheet :324-332) to sheet_path and one Snapshot2 record
 * (OutputPanels :317-322) to result_path; NULL or "" writes none.  Records
 * are the protobuf wire format of proto/uvlm.proto, each preceded by its
 * byte length as a little-endian uint64.  The state is snapshotted on the
 * device and written by a background thread; uvlm_flush_output waits for
 * it, uvlm_destroy flushes and closes.  Calling again replaces the files. */
#define UVLM_OUTPUT_SHEETS 0
#define UVLM_OUTPUT_SNAPSHOT2 1
int uvlm_set_output_paths(uvlm_ctx* ctx, const char* sheet_path, const char* result_path);
int uvlm_flush_output(uvlm_ctx* ctx);
/* One record of `kind` from host arrays in the simulator's layout (wing
 * nodes [num][rows+1][cols+1][3], circulations [num][rows][cols], wake
 * nodes [num][wake_rows+1][cols+1][3], circulations [num][wake_rows][cols]),
 * appended to (append = 1) or replacing the file at path. */
int uvlm_write_state_record(const char* path, int32_t append, int32_t kind, int64_t num, int64_t rows, int64_t cols,
                            int64_t wake_rows, const double* wing_pos, const double* wing_gamma,
                            const double* wake_pos, const double* wake_gamma, double t);
/* The legacy simulator's per-step file (OutputSnapshot2,
 * src/simulator/simulator.cpp:118-160): one Snapshot2 message, unframed
 * (SerializeToOstream), replacing the file at path.  It holds t; one
 * ContainerShape per container (rows, cols, id = its index, chord, span);
 * one VortexRing per ring of the pool (rings and reference nodes rings0
 * [n_rings][4][3], rings0 NULL writes no nodes0; gamma [n_rings]); and
 * n_mv MorphingVelocity records (center [3], the four segment velocities
 * [4][3], freestream [3] each). */
int uvlm_write_legacy_snapshot2(const char* path, double t, int64_t n_containers, const int64_t* rows,
                                const int64_t* cols, const double* chord, const double* span, const double* rings,
                                const double* rings0, const double* gamma, int64_t n_rings, const double* mv_center,
                                const double* mv_nodes, const double* mv_freestream, int64_t n_mv);

/* ---------------------------------------------- learned warm start (MLP) */
/* No counterpart in the reference.  A per-panel MLP (8 features -> 3 x 256
 * GELU -> 1, BF16 weights, FP32 accumulation) predicts the correction of the
 * extrapolation 2*G_n - G_{n-1} of each panel's circulation from
 * (G_n, G_n - G_{n-1}, b_{n+1}, b_{n+1} - b_n, sin/cos of the dominant
 * kinematic phase, chordwise/spanwise position); the result seeds the GMRES
 * solve when cfg.warm_start == UVLM_WARM_MLP. */
typedef struct uvlm_mlp uvlm_mlp;
int uvlm_mlp_create(uint64_t seed, uvlm_mlp** out);
int uvlm_mlp_destroy(uvlm_mlp* mlp);
int64_t uvlm_mlp_num_params(const uvlm_mlp* mlp);
/* FP32 master parameters: per layer W [in][out] then b [out]. */
int uvlm_mlp_get_params(const uvlm_mlp* mlp, float* params);
int uvlm_mlp_set_params(uvlm_mlp* mlp, const float* params);
/* x' = (x - mean) / stdev per feature; prediction = out_scale * network(x'). */
int uvlm_mlp_set_normalization(uvlm_mlp* mlp, const float* mean, const float* stdev, float out_scale);
/* Host arrays: x [n][8], y [n]. */
int uvlm_mlp_forward(uvlm_mlp* mlp, const float* x, int64_t n, float* y);
/* The same network on the tcgen05 tensor cores (the inference the time-
 * stepper uses for UVLM_WARM_MLP): the hidden layers take BF16 activations
 * and BF16 weights with FP32 accumulation in TMEM, so y differs from
 * uvlm_mlp_forward (FP32 activations) at the BF16 level.  UVLM_ERR_UNSUPPORTED
 * off sm_100 devices. */
int uvlm_mlp_forward_tc(uvlm_mlp* mlp, const float* x, int64_t n, float* y);
/* Mean-square loss on (prediction - target)/out_scale and its gradient with
 * respect to every parameter (same layout as the parameters). */
int uvlm_mlp_gradients(uvlm_mlp* mlp, const float* x, const float* target, int64_t n, float* grads, double* loss);
/* Adam on shuffled minibatches; final_loss = mean loss of the last epoch. */
int uvlm_mlp_train(uvlm_mlp* mlp, const float* x, const float* target, int64_t n, int32_t epochs, int32_t batch,
                   double lr, uint64_t seed, double* final_loss);
/* The context uses (borrows) this network for UVLM_WARM_MLP. */
int uvlm_set_mlp(uvlm_ctx* ctx, uvlm_mlp* mlp);
/* Record (features, target) pairs of every solve from step 2 on, up to
 * max_samples panels (enable = 0 frees the buffer). */
int uvlm_collect_training_data(uvlm_ctx* ctx, int32_t enable, int64_t max_samples);
/* n = samples recorded; X [n][8] and T [n] (either may be NULL). */
int uvlm_get_training_data(uvlm_ctx* ctx, float* X, float* T, int64_t* n);

/* FP32 LU with partial pivoting of a row-major n x n matrix (host arrays);
 * update: 0 SIMT FP32, 1 tcgen05 TF32, 2 tcgen05 BF16 trailing updates.  LU
 * receives L (unit diagonal, below) and U; ipiv the LAPACK-style row swaps
 * (0-based).  The factorisation stage of the mixed-precision solve. */
int uvlm_lu_factor_f32(const float* A, int64_t n, int32_t update, float* LU, int32_t* ipiv);
/* Dense solve A x = b, A row-major n x n (FullPivLU replacement).  method:
 * 0 FP64 LU; 1 TF32 LU + FP64-residual GMRES; 2 BF16 LU + GMRES.
 * iters (may be NULL) receives the GMRES iteration count. */
int uvlm_dense_solve(const double* A, int64_t n, const double* b, double* x, int32_t method, int32_t* iters);

/* ---------------------------------------------------------------------------
 * Batched independent cases (no counterpart in the reference, whose drivers
 * run one SimpleSimulator per process).  Every case is one wing with its own
 * lattice, kinematics, forward flight and dt; all cases advance together, one
 * MainLoop (simple_simulator.cpp:240-286) per step: kinematics, shed,
 * influence matrix, RHS, solve, Joukowski loads, advection.  Each stage is one
 * launch over all cases (persistent N-body over (case, target tile, source
 * split) items, one CTA per case for the dense solve), the stage sizes are
 * derived on the device from a step counter, and one step is captured as a
 * CUDA graph that every further step replays.
 * ------------------------------------------------------------------------- */
typedef struct uvlm_batch uvlm_batch;

typedef struct {
  double chord, span;
  int64_t rows, cols;        /* rings chordwise x spanwise (cols even; rows, cols <= 64, rows*cols <= 1024) */
  double origin[3];          /* wing origin (also the Morphing origin) */
  double forward_flight[3];  /* SimpleSimulator::set_forward_flight */
  double dt;                 /* this case's time step; t = step * dt */
  uvlm_kinematics kin;       /* origin is overwritten with the wing origin */
  int32_t chebyshev_chord, chebyshev_span;
} uvlm_batch_case;

typedef struct {
  int32_t precision;       /* FP64: FP64 N-body and LU; MIXED: FP32 N-body, FP32 LU with FP64 iterative
                              refinement (residual b - A g with the FP64 matrix) */
  int32_t advection;       /* UVLM_ADVECT_EULER or UVLM_ADVECT_RK2 */
  int32_t rk_ignore_rows;  /* RK2: Euler for wake rows i <= this (5, src/advect.h:77) */
  int32_t refine_max_iter; /* MIXED: refinement sweeps at most */
  double refine_tol;       /* MIXED: stop when ||b - A g|| <= tol ||b|| */
  int64_t max_steps;       /* MainLoops the batch can run (wake capacity) */
  int32_t device;
  int32_t use_graph;       /* 1: capture one step as a CUDA graph and replay it */
  int32_t stale_factors;   /* MIXED, 1: a case refines from its previous circulation with the FP32 factors
                              of an earlier step and is factored again only when that does not converge */
  int32_t nbody_tile;      /* MIXED: -1 (default) the tile autotuner picks the N-body tile at creation, timing
                              every compiled FP32 tile on the last step's advection over a synthetic wake;
                              0..2 pins a tile (see uvlm_batch_nbody_tile_name) */
} uvlm_batch_config;

int uvlm_batch_config_default(uvlm_batch_config* cfg);
int uvlm_batch_create(const uvlm_batch_config* cfg, const uvlm_batch_case* cases, int32_t n_cases,
                      uvlm_batch** out);
int uvlm_batch_destroy(uvlm_batch* b);
const char* uvlm_batch_last_error(const uvlm_batch* b);
/* n_steps more MainLoops of every case (step = steps_done, steps_done+1, ...). */
int uvlm_batch_run(uvlm_batch* b, int64_t n_steps);
int uvlm_batch_steps_done(const uvlm_batch* b, int64_t* steps);
/* rows [steps_done][n_cases][3] = (t, CD, CL) of every MainLoop so far. */
int uvlm_batch_get_loads(const uvlm_batch* b, double* rows);
/* State of case c (any pointer may be NULL): wing_pos [(rows+1)(cols+1)][3],
 * wing_gamma [rows][cols], wake_pos [wake_rows+1][cols+1][3] (row 0 newest),
 * wake_gamma [wake_rows][cols]. */
int uvlm_batch_get_case(const uvlm_batch* b, int32_t c, double* wing_pos, double* wing_gamma, double* wake_pos,
                        double* wake_gamma, int64_t* wake_rows);
/* Last step's solve per case: refinement sweeps and final relative residual. */
int uvlm_batch_get_solve_stats(const uvlm_batch* b, int32_t* sweeps, double* residual);
/* Per-case factorisations so far (every case every step when stale_factors = 0). */
int uvlm_batch_factorizations(const uvlm_batch* b, int64_t* count);
/* Kernels one step launches (nodes of the captured graph). */
int uvlm_batch_launches_per_step(const uvlm_batch* b, int64_t* launches);
/* Name of the N-body tile the batch runs (chosen by the autotuner or pinned). */
const char* uvlm_batch_nbody_tile_name(const uvlm_batch* b);
/* The batch's CUDA stream (a cudaStream_t), for events around uvlm_batch_run. */
void* uvlm_batch_stream(const uvlm_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* UVLM_B200_H_ */
