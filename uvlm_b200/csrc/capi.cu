// capi.cu -- the C-ABI: context, SimpleSimulator::MainLoop orchestration on
// the device, and the context-free replacements of the reference API.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/uvlm_b200.h"
#include "gmres.cuh"
#include "host_lattice.h"
#include "mlp.cuh"
#include "lu.cuh"
#include "nbody.cuh"
#include "output.cuh"
#include "step.cuh"

using namespace uvlm;

namespace {

thread_local std::string g_last_error;

}  // namespace

void uvlm::set_global_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<long long> g_launches{0};
void uvlm::note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {

int set_global(const Error& e) {
  if (e.code) g_last_error = e.msg;
  return e.code;
}

template <class T>
Error dalloc(T** p, size_t count) {
  if (*p) cudaFree(*p);
  *p = nullptr;
  if (count == 0) return ok();
  UVLM_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count));
  return ok();
}

int device_sms(int dev) {
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  return v;
}

}  // namespace

namespace uvlm {
Mlp* mlp_of(uvlm_mlp* h);
}

struct uvlm_ctx {
  uvlm_config cfg{};
  std::vector<uvlm_wing_desc> wings;
  std::vector<std::vector<double>> wing_nodes;  // per wing: the caller's lattice, or empty (RectGenerator)
  std::vector<uvlm_kinematics> kins;
  double ff[3] = {0, 0, 0};
  std::string err;
  cudaStream_t st = nullptr;
  int num_sms = 148;
  bool built = false;
  bool timing = false;

  int num = 0, R = 0, C = 0, N = 0;
  int PR = 0;            // physical node rows per wake sheet
  int wake_start = 0;    // physical row of logical node row 0
  int wake_nodes = 0;    // logical node rows (0 before the first shed)
  bool has_vprev = false;
  long long tcap = 0;

  uvlm_kinematics* d_kin = nullptr;
  double* d_chord_span = nullptr;
  double *d_pos_init = nullptr, *d_pos = nullptr;
  double *d_gamma = nullptr, *d_gamma_prev = nullptr, *d_gamma_hist = nullptr;
  double *d_wpos = nullptr, *d_wpos2 = nullptr, *d_wgamma = nullptr;
  double *d_k1 = nullptr, *d_k2 = nullptr, *d_k3 = nullptr, *d_vprev = nullptr;
  double *d_cx = nullptr, *d_cy = nullptr, *d_cz = nullptr, *d_normal = nullptr, *d_area = nullptr, *d_uls = nullptr;
  double* d_rhs = nullptr;
  double* d_line_uls = nullptr;
  double *d_tx = nullptr, *d_ty = nullptr, *d_tz = nullptr, *d_vx = nullptr, *d_vy = nullptr, *d_vz = nullptr;
  double* d_A64 = nullptr;   // FP64 matrix (plain: factored in place; mixed: residual matrix if assembly_fp64)
  float* d_A32 = nullptr;    // FP32 matrix of the mixed form
  float* d_F32 = nullptr;    // FP32 factors of the mixed form
  float* d_Minv = nullptr;   // dense (LU)^-1 of those factors, applied after their row permutation (UVLM_PRECOND_INVERSE)
  double* d_F64 = nullptr;   // mixed form: FP64 factors of the fallback solve (a copy of d_A64)
  LuWork lu64;               // ... and its pivots and scratch
  double* d_tmp = nullptr;   // [N] scratch
  double* d_row = nullptr;   // [1+2num] load row
  int* d_flags = nullptr;    // [4] non-finite etc.
  double* h_row = nullptr;   // pinned
  int* h_flags = nullptr;    // pinned
  NBodyWork nb;
  LuWork lu;
  GmresWork gm;
  bool have_factors = false;
  bool refresh_next = false;  // refactor at the next solve (GMRES reached gmres_refresh_iter)
  // N-body tile variant per stage (kStageRhs, kStageLoads, kStageAdvect) and
  // precision ([0] FP32, [1] FP64); defaults fp32_h3_t2_b128_x2f and
  // fp64_h2_t1_b128_m3, each autotuned on that stage's first large evaluation
  // unless the configuration pins one
  int stage_variant[3][2] = {{16, 9}, {16, 9}, {16, 9}};
  bool stage_pinned[3][2] = {};        // the configuration chose the tile
  double stage_tuned_pairs[3][2] = {};  // pairs of the evaluation the tile was tuned on (0: not yet)
  // learned warm start: network (borrowed), per-step features, collected data
  uvlm_mlp* mlp = nullptr;
  double* d_rhs_prev = nullptr;
  double* d_phase = nullptr;
  double* h_phase = nullptr;
  float* d_feat = nullptr;
  float* d_mlp_y = nullptr;
  bool collect = false;
  long long collect_cap = 0, collect_n = 0;
  float* d_collect_x = nullptr;
  float* d_collect_t = nullptr;
  Error warm_phase(double t);
  Error warm_features(double t);
  bool mlp_tc_used = false;  // this step's guess came from the tensor-core inference
  uvlm_step_stats last{};
  double work_nbody = 0, work_asm = 0, work_lu = 0;
  cudaEvent_t ev[8] = {};
  // per-launch events around the N-body evaluations of a timed step
  static constexpr int kNbEvents = 8;
  cudaEvent_t nbev[2 * kNbEvents] = {};
  int nbev_n = 0;
  cudaEvent_t fev[3] = {};  // around the FP32 LU and the dense inverse of a refactorisation
  bool fev_used = false;
  OutputWriter* out = nullptr;  // per-step AllVortexSheets / Snapshot2 records

  WingShape ws() const { return WingShape{num, R, C}; }
  WakeLayout wl() const { return WakeLayout{num, C, PR, wake_start, wake_nodes}; }
  int wake_rings() const { return wake_nodes > 0 ? wake_nodes - 1 : 0; }
  bool mixed() const { return cfg.precision == UVLM_PRECISION_MIXED; }

  int fail_with(const Error& e) {
    if (e.code) err = e.msg;
    return e.code;
  }
  void free_all();
  Error alloc_all();
  // precision of an N-body stage (UVLM_STAGE_* bit): the context's, or FP64
  // where the mixed form is told to evaluate that stage in FP64
  NBodyPrec stage_prec(int stage_bit) const {
    return (!mixed() || (cfg.nbody_fp64_stages & stage_bit)) ? kNBodyFP64 : kNBodyFP32;
  }
  // whether the FP32 evaluation of a stage takes its near pairs in FP64
  bool stage_near64(int stage_bit) const { return mixed() && (cfg.nbody_near_fp64 & stage_bit) != 0; }
  Error build_sources(bool with_bound, const double* wake_pos_buf, NBodyPrec prec, SourceBlock* blocks, int* nb_out);
  static constexpr int kStageRhs = 0, kStageLoads = 1, kStageAdvect = 2;
  Error eval(const SourceBlock* blocks, int nblocks, long long nt, NBodyPrec prec, int stage);
  Error shed(long long step);
  Error solve(long long step);
  Error advect(double dt);
  Error step(long long step, double dt, double* row);
  // MainLoop in stages (uvlm_step runs all six in order)
  Error stage_kinematics(long long step, double dt);
  Error stage_assemble();
  Error stage_rhs();
  Error stage_solve();
  Error stage_loads();
  Error stage_advect(double* row);
  int stage_next = 0;  // the stage a staged MainLoop expects next (0: none in progress)
  long long stage_step = 0;
  double cur_dt = 0;
  void mark(int i) {
    if (timing) cudaEventRecord(ev[i], st);
  }
};

void uvlm_ctx::free_all() {
  double** dd[] = {&d_pos_init, &d_pos, &d_gamma, &d_gamma_prev, &d_gamma_hist, &d_wpos, &d_wpos2, &d_wgamma, &d_k1, &d_k2,
                   &d_k3, &d_vprev, &d_cx, &d_cy, &d_cz, &d_normal, &d_area, &d_uls, &d_rhs, &d_line_uls,
                   &d_tx, &d_ty, &d_tz, &d_vx, &d_vy, &d_vz, &d_A64, &d_tmp, &d_row, &d_chord_span};
  for (auto p : dd) {
    cudaFree(*p);
    *p = nullptr;
  }
  cudaFree(d_A32);
  cudaFree(d_F32);
  cudaFree(d_Minv);
  d_Minv = nullptr;
  cudaFree(d_F64);
  d_F64 = nullptr;
  lu_work_free(&lu64);
  cudaFree(d_rhs_prev);
  cudaFree(d_phase);
  cudaFree(d_feat);
  cudaFree(d_mlp_y);
  if (h_phase) cudaFreeHost(h_phase);
  d_rhs_prev = d_phase = nullptr;
  h_phase = nullptr;
  d_feat = d_mlp_y = nullptr;
  cudaFree(d_kin);
  cudaFree(d_flags);
  cudaFree(nb.records);
  cudaFree(nb.partial);
  cudaFree(nb.records64);
  d_A32 = d_F32 = nullptr;
  d_kin = nullptr;
  d_flags = nullptr;
  nb = NBodyWork{};
  if (h_row) cudaFreeHost(h_row);
  if (h_flags) cudaFreeHost(h_flags);
  h_row = nullptr;
  h_flags = nullptr;
  lu_work_free(&lu);
  gmres_work_free(&gm);
  have_factors = false;
}

Error uvlm_ctx::alloc_all() {
  free_all();
  const size_t nn = (size_t)num * (R + 1) * (C + 1);
  const size_t wn = (size_t)num * PR * (C + 1);
  UVLM_TRY(dalloc(&d_kin, (size_t)num));
  UVLM_TRY(dalloc(&d_chord_span, (size_t)2 * num));
  UVLM_TRY(dalloc(&d_pos_init, 3 * nn));
  UVLM_TRY(dalloc(&d_pos, 3 * nn));
  UVLM_TRY(dalloc(&d_gamma, (size_t)N));
  UVLM_TRY(dalloc(&d_gamma_prev, (size_t)N));
  UVLM_TRY(dalloc(&d_gamma_hist, (size_t)N));
  for (double** p : {&d_wpos, &d_wpos2, &d_k1, &d_k2, &d_k3, &d_vprev}) UVLM_TRY(dalloc(p, 3 * wn));
  UVLM_TRY(dalloc(&d_wgamma, (size_t)num * PR * C));
  for (double** p : {&d_cx, &d_cy, &d_cz, &d_area, &d_rhs, &d_tmp}) UVLM_TRY(dalloc(p, (size_t)N));
  UVLM_TRY(dalloc(&d_normal, 3 * (size_t)N));
  UVLM_TRY(dalloc(&d_uls, 3 * (size_t)N));
  const long long lines = (long long)num * R * (2 * C + 1);
  tcap = std::max<long long>({(long long)N, lines, (long long)wn});
  UVLM_TRY(dalloc(&d_line_uls, 3 * (size_t)lines));
  for (double** p : {&d_tx, &d_ty, &d_tz, &d_vx, &d_vy, &d_vz}) UVLM_TRY(dalloc(p, (size_t)tcap));
  UVLM_TRY(dalloc(&d_row, (size_t)(1 + 2 * num)));
  UVLM_TRY(dalloc(&d_rhs_prev, (size_t)N));
  UVLM_TRY(dalloc(&d_phase, (size_t)num));
  UVLM_TRY(dalloc(&d_feat, (size_t)N * kMlpIn));
  UVLM_TRY(dalloc(&d_mlp_y, (size_t)N));
  UVLM_CUDA_TRY(cudaMallocHost(&h_phase, sizeof(double) * num));
  UVLM_CUDA_TRY(cudaMemset(d_rhs_prev, 0, sizeof(double) * N));
  UVLM_TRY(dalloc(&d_flags, 4));
  UVLM_CUDA_TRY(cudaMallocHost(&h_row, sizeof(double) * (1 + 2 * num)));
  UVLM_CUDA_TRY(cudaMallocHost(&h_flags, sizeof(int) * 12));
  // N-body scratch: records for bound + wake sheets, per-split partial sums
  nb.records_cap = (long long)(nn + wn) * (long long)sizeof(RecD);
  UVLM_CUDA_TRY(cudaMalloc(&nb.records, nb.records_cap));
  nb.partial_cap = 3LL * std::max<long long>(64LL * N, 16LL * tcap);
  UVLM_CUDA_TRY(cudaMalloc(&nb.partial, sizeof(double) * nb.partial_cap));
  if (mixed() && cfg.nbody_near_fp64) {
    nb.records64_cap = (long long)(nn + wn) * (long long)sizeof(RecD);
    UVLM_CUDA_TRY(cudaMalloc(&nb.records64, nb.records64_cap));
  }
  // dense matrices
  if (!mixed() || cfg.assembly_fp64) UVLM_TRY(dalloc(&d_A64, (size_t)N * N));
  if (mixed()) {
    if (!cfg.assembly_fp64) UVLM_CUDA_TRY(cudaMalloc(&d_A32, sizeof(float) * (size_t)N * N));
    UVLM_CUDA_TRY(cudaMalloc(&d_F32, sizeof(float) * (size_t)N * N));
    if (cfg.solver == UVLM_SOLVER_GMRES_STALE && cfg.preconditioner == UVLM_PRECOND_INVERSE)
      UVLM_CUDA_TRY(cudaMalloc(&d_Minv, sizeof(float) * (size_t)N * N));
    UVLM_TRY(lu_work_alloc(&lu, N, 4, num_sms));
    lu.local_pivot = cfg.lu_pivoting == UVLM_PIVOT_LOCAL;
    UVLM_TRY(gmres_work_alloc(&gm, N, std::max(2, cfg.gmres_restart)));
    if (cfg.assembly_fp64) {  // the plain fresh-LU solve that backs up the GMRES solve
      UVLM_TRY(dalloc(&d_F64, (size_t)N * N));
      UVLM_TRY(lu_work_alloc(&lu64, N, 8, num_sms));
    }
  } else {
    UVLM_TRY(lu_work_alloc(&lu, N, 8, num_sms));
  }
  std::vector<double> cs;
  for (auto& w : wings) {
    cs.push_back(w.chord);
    cs.push_back(w.span);
  }
  UVLM_CUDA_TRY(cudaMemcpy(d_chord_span, cs.data(), sizeof(double) * cs.size(), cudaMemcpyHostToDevice));
  return ok();
}

// Source records: [bound sheets][wake sheets (positions from wake_pos_buf)].
Error uvlm_ctx::build_sources(bool with_bound, const double* wake_pos_buf, NBodyPrec prec, SourceBlock* blocks,
                              int* nb_out) {
  SheetView views[2];
  int nv = 0;
  if (with_bound) views[nv++] = SheetView{d_pos, R + 1, 0, d_gamma, R, 0, num, R + 1, C};
  if (wake_rings() > 0)
    views[nv++] = SheetView{wake_pos_buf, PR, wake_start, d_wgamma, PR, wake_start, num, wake_nodes, C};
  *nb_out = nv;
  if (nv == 0) return ok();
  return nbody_build_sources(views, nv, prec, &nb, blocks, st);
}

Error uvlm_ctx::eval(const SourceBlock* blocks, int nblocks, long long nt, NBodyPrec prec, int stage) {
  const double pairs = (double)nt * (double)nbody_unique_segments(blocks, nblocks);
  work_nbody += pairs;
  const int pi = prec == kNBodyFP64 ? 1 : 0;
  int& chosen = stage_variant[stage][pi];
  // tune on the first evaluation with >= 2e9 pairs and again whenever the
  // stage has grown by half since (a growing wake changes the far-strip share)
  if (!stage_pinned[stage][pi] && nblocks > 0 && pairs >= 2e9 && pairs >= 1.5 * stage_tuned_pairs[stage][pi]) {
    // Tile autotune on the stage's first large evaluation: time every
    // compiled variant of this precision on the real sources and targets,
    // keep the fastest (the default unless another is more than 3% faster).
    // The stages differ in their targets (collocation points, load lines,
    // wake nodes), and so in the share of far strips the walkers skip.
    float best_ms = 1e30f;
    int best = chosen;
    for (int v = 0; v < nbody_num_variants(); ++v) {
      if (nbody_variant_prec(v) != prec) continue;
      if (prec == kNBodyFP32 && cfg.nbody_near_fp64 && !nbody_variant_near64(v)) continue;  // keep the FP64 near field
      float ms = 0;
      for (int rep = 0; rep < 2; ++rep) {
        UVLM_CUDA_TRY(cudaEventRecord(ev[0], st));
        UVLM_TRY(nbody_eval(blocks, nblocks, prec, d_tx, d_ty, d_tz, nt, d_vx, d_vy, d_vz, &nb, v, num_sms, st));
        UVLM_CUDA_TRY(cudaEventRecord(ev[1], st));
        UVLM_CUDA_TRY(cudaEventSynchronize(ev[1]));
        UVLM_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
      }
      const bool is_default = v == chosen;
      const float score = is_default ? ms / 1.03f : ms;
      if (score < best_ms) {
        best_ms = score;
        best = v;
      }
    }
    chosen = best;
    stage_tuned_pairs[stage][pi] = pairs;
  }
  if (nblocks == 0) {
    UVLM_CUDA_TRY(cudaMemsetAsync(d_vx, 0, sizeof(double) * nt, st));
    UVLM_CUDA_TRY(cudaMemsetAsync(d_vy, 0, sizeof(double) * nt, st));
    UVLM_CUDA_TRY(cudaMemsetAsync(d_vz, 0, sizeof(double) * nt, st));
    return ok();
  }
const bool rec = timing && nbev_n < kNbEvents;
  if (rec) UVLM_CUDA_TRY(cudaEventRecord(nbev[2 * nbev_n], st));
  const Error e = nbody_eval(blocks, nblocks, prec, d_tx, d_ty, d_tz, nt, d_vx, d_vy, d_vz, &nb,
                             chosen, num_sms, st);
  if (rec) {
    UVLM_CUDA_TRY(cudaEventRecord(nbev[2 * nbev_n + 1], st));
    ++nbev_n;
  }
  return e;
}

Error uvlm_ctx::shed(long long step) {
  if (wake_start == 0) {
    // compact the prepend buffer: move the live rows to the end
    const int to = PR - wake_nodes;
    if (to <= 0) return fail(kErrCapacity, "wake longer than max_wake_rows");
    UVLM_TRY(launch_move_rows(d_wpos, num, PR, 3 * (C + 1), wake_start, to, wake_nodes, d_k3, st));
    UVLM_TRY(launch_move_rows(d_wgamma, num, PR, C, wake_start, to, wake_nodes, d_k3, st));
    if (has_vprev) UVLM_TRY(launch_move_rows(d_vprev, num, PR, 3 * (C + 1), wake_start, to, wake_nodes, d_k3, st));
    wake_start = to;
  }
  wake_start -= 1;
  wake_nodes += 1;
  return launch_shed(ws(), d_pos, d_gamma, wl(), d_wpos, d_wgamma, step > 0, st);
}

Error uvlm_ctx::solve(long long step) {
  last.refactored = 0;
  last.gmres_iters = 0;
  last.residual = 0;
  if (!mixed()) {
    // plain form: FP64 assembly, fresh FP64 LU, FP64 triangular solves
    UVLM_TRY(lu_factor_f64(d_A64, N, &lu, st));
    UVLM_TRY(lu_solve_f64(d_A64, N, &lu, d_rhs, d_gamma, d_tmp, st));
    last.solve_path = 0;
    last.refactored = 1;
    work_lu += 2.0 / 3.0 * (double)N * N * N;
    return ok();
  }
  const LuUpdate upd = cfg.lu_precision == UVLM_LU_BF16 ? kLuUpdateBF16 : kLuUpdateTF32;
  const LuUpdate use = gemm_tc_available() ? upd : kLuUpdateSimt;
  auto factor = [&]() -> Error {
    if (cfg.assembly_fp64)
      UVLM_TRY(launch_assemble(ws(), d_pos, d_cx, d_cy, d_cz, d_normal, true, d_F32, true, st));
    else
      UVLM_CUDA_TRY(cudaMemcpyAsync(d_F32, d_A32, sizeof(float) * (size_t)N * N, cudaMemcpyDeviceToDevice, st));
    if (timing && fev[0]) UVLM_CUDA_TRY(cudaEventRecord(fev[0], st));
    UVLM_TRY(lu_factor_f32(d_F32, N, use, &lu, st));
    UVLM_TRY(lu_check(&lu, st));
    if (timing && fev[1]) UVLM_CUDA_TRY(cudaEventRecord(fev[1], st));
    if (d_Minv) UVLM_TRY(lu_inverse_f32(d_F32, N, use, &lu, d_Minv, st));
    if (timing && fev[2]) {
      UVLM_CUDA_TRY(cudaEventRecord(fev[2], st));
      fev_used = true;
    }
    have_factors = true;
    last.refactored = 1;
    work_lu += 2.0 / 3.0 * (double)N * N * N;
    return ok();
  };
  // a fresh factorisation every step (the LU solver), on the first step, or
  // when the previous step's GMRES needed gmres_refresh_iter iterations or more
  const bool fresh = cfg.solver == UVLM_SOLVER_LU || !have_factors || refresh_next;
  refresh_next = false;
  if (fresh) UVLM_TRY(factor());
  // initial guess: d_gamma holds g_n (the previous solution); the linear
  // extrapolation 2 g_n - g_{n-1} uses the history kept in d_gamma_hist
  if (cfg.warm_start == UVLM_WARM_EXTRAPOLATE && step >= 2)
    UVLM_TRY(launch_extrapolate(d_gamma, d_gamma_prev, d_gamma_hist, N, st));
  if (cfg.warm_start == UVLM_WARM_MLP && step >= 2) {
    if (!mlp) return fail(kErrState, "warm_start MLP needs uvlm_set_mlp");
    if (mlp_tc_available()) {
      // features, the three hidden layers on the tensor cores, the head and
      // the guess in one kernel
      UVLM_TRY(warm_phase(step * cur_dt));
      UVLM_TRY(mlp_guess_tc(mlp_of(mlp), num, R, C, d_gamma_prev, d_gamma_hist, d_rhs, d_rhs_prev, d_phase, d_gamma,
                            st));
      mlp_tc_used = true;
    } else {
      UVLM_TRY(warm_features(step * cur_dt));
      UVLM_TRY(mlp_forward(mlp_of(mlp), d_feat, N, d_mlp_y, st));
      UVLM_TRY(mlp_apply_guess(N, d_gamma_prev, d_gamma_hist, d_mlp_y, d_gamma, st));
    }
  }
  const float* A32 = cfg.assembly_fp64 ? nullptr : d_A32;
  const double* A64 = cfg.assembly_fp64 ? d_A64 : nullptr;
  GmresResult r;
  UVLM_TRY(gmres_solve(A32, A64, N, d_F32, &lu, d_Minv, d_rhs, d_gamma, cfg.gmres_tol, cfg.gmres_max_iter, &gm, &r, st));
  last.solve_path = fresh ? 0 : 1;
  last.gmres_iters = r.iters;
  last.initial_residual = r.initial_relres;
  if (!r.converged) {
    // More than gmres_max_iter iterations (or a non-finite initial guess):
    // the plain fresh-LU solve, an FP64 LU of the FP64 matrix of this step,
    // gives the circulation (the plain form's own solve, which also judges
    // the error of the accelerated path); the FP32 factors are refreshed so
    // that the next steps' GMRES is preconditioned by this step's matrix.
    last.solve_path = 2;
    if (!fresh) UVLM_TRY(factor());
    if (d_F64) {
      UVLM_CUDA_TRY(cudaMemcpyAsync(d_F64, d_A64, sizeof(double) * (size_t)N * N, cudaMemcpyDeviceToDevice, st));
      UVLM_TRY(lu_factor_f64(d_F64, N, &lu64, st));
      UVLM_TRY(lu_check(&lu64, st));
      UVLM_TRY(lu_solve_f64(d_F64, N, &lu64, d_rhs, d_gamma, d_tmp, st));
      UVLM_TRY(lu_check(&lu64, st));
      work_lu += 2.0 / 3.0 * (double)N * N * N;
      // residual of the plain solve (zero GMRES iterations from its answer)
      GmresResult rp;
      UVLM_TRY(gmres_solve(A32, A64, N, d_F32, &lu, d_Minv, d_rhs, d_gamma, 1.0, 0, &gm, &rp, st));
      last.residual = rp.relres;
      return ok();
    }
    // FP32 assembly only (no FP64 matrix): a fresh FP32 factorisation and GMRES again
    UVLM_CUDA_TRY(cudaMemcpyAsync(d_gamma, d_gamma_prev, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    GmresResult r2;
    UVLM_TRY(gmres_solve(A32, A64, N, d_F32, &lu, d_Minv, d_rhs, d_gamma, cfg.gmres_tol, 4 * cfg.gmres_max_iter, &gm, &r2,
                         st));
    last.gmres_iters += r2.iters;
    r = r2;
  }
  last.residual = r.relres;
  if (!r.converged) return fail(kErrNonFinite, "GMRES did not converge after a fresh factorisation");
  // aging factors: refactor from the next step's matrix before GMRES reaches its cap (the fallback
  // costs a fresh FP64 LU on top of the refactorisation)
  if (!fresh && cfg.gmres_refresh_iter > 0 && r.iters >= cfg.gmres_refresh_iter) refresh_next = true;
  return ok();
}

Error uvlm_ctx::advect(double dt) {
  const WakeLayout L = wl();
  SourceBlock blocks[2];
  int nbk = 0;
  const NBodyPrec prec = stage_prec(UVLM_STAGE_ADVECT);
  nb.near64 = stage_near64(UVLM_STAGE_ADVECT);
  // velocities at the wake rows first_row.. (sources: bound and wake sheets at pos_buf)
  auto velocity_at = [&](const double* pos_buf, bool rebuild, int first_row) -> Error {
    if (rebuild) UVLM_TRY(build_sources(true, pos_buf, prec, blocks, &nbk));
    const long long n_rows = std::max(0, wake_nodes - first_row);
    const long long n_tgt = (long long)num * n_rows * (C + 1);
    if (n_tgt > 0) {
      UVLM_TRY(launch_gather_wake(L, pos_buf, d_tx, d_ty, d_tz, st, first_row));
      UVLM_TRY(eval(blocks, nbk, n_tgt, prec, kStageAdvect));
    }
    return ok();
  };
  const int ign = cfg.rk_ignore_rows;
  // The last evaluation of RK2 and of RK4 only feeds the rows past ignore_rows (the others take the
  // Euler step, src/advect.cpp:71-79, :167-178): its targets start there.  The earlier RK4
  // evaluations move the whole intermediate wake (the sources of the next one) and take every row.
  const int rk2_row0 = std::max(1, ign + 1);
  const bool loads_built = cfg.compute_loads != 0;
  switch (cfg.advection) {
    case UVLM_ADVECT_EULER:
      UVLM_TRY(velocity_at(d_wpos, true, 1));
      UVLM_TRY(launch_advect(kAdvEuler, L, d_wpos, d_wpos2, d_k1, d_k2, d_k3, d_vprev, false, d_vx, d_vy, d_vz, ff, dt,
                             ign, st));
      break;
    case UVLM_ADVECT_RK2:
      UVLM_TRY(velocity_at(d_wpos, true, 1));
      UVLM_TRY(launch_advect(kAdvRK2K1, L, d_wpos, d_wpos2, d_k1, d_k2, d_k3, d_vprev, false, d_vx, d_vy, d_vz, ff, dt,
                             ign, st));
      UVLM_TRY(velocity_at(d_wpos2, true, rk2_row0));
      UVLM_TRY(launch_advect(kAdvRK2Upd, L, d_wpos, d_wpos2, d_k1, d_k2, d_k3, d_vprev, false, d_vx, d_vy, d_vz, ff,
                             dt, ign, st, rk2_row0));
      break;
    case UVLM_ADVECT_RK4:
      UVLM_TRY(velocity_at(d_wpos, true, 1));
      UVLM_TRY(launch_advect(kAdvRK4K1, L, d_wpos, d_wpos2, d_k1, d_k2, d_k3, d_vprev, false, d_vx, d_vy, d_vz, ff, dt,
                             ign, st));
      UVLM_TRY(velocity_at(d_wpos2, true, 1));
      UVLM_TRY(launch_advect(kAdvRK4K2, L, d_wpos, d_wpos2, d_k1, d_k2, d_k3, d_vprev, false, d_vx, d_vy, d_vz, ff, dt,
                             ign, st));
      UVLM_TRY(velocity_at(d_wpos2, true, rk2_row0));
      UVLM_TRY(launch_advect(kAdvRK4Upd, L, d_wpos, d_wpos2, d_k1, d_k2, d_k3, d_vprev, false, d_vx, d_vy, d_vz, ff,
                             dt, ign, st, rk2_row0));
      break;
    case UVLM_ADVECT_AB2:
      UVLM_TRY(velocity_at(d_wpos, true, 1));
      UVLM_TRY(launch_advect(kAdvAB2, L, d_wpos, d_wpos2, d_k1, d_k2, d_k3, d_vprev, has_vprev, d_vx, d_vy, d_vz, ff,
                             dt, ign, st));
      has_vprev = true;
      break;
    default:
      return fail(kErrInvalid, "unknown advection scheme");
  }
  (void)loads_built;
  return ok();
}

// Features of the learned warm start for the solve at time t: G_n (the
// previous solution), G_{n-1}, the new and the previous RHS and the phase of
// each wing's dominant motion (first non-zero angular frequency of plug,
// flap, twist, bend).
Error uvlm_ctx::warm_phase(double t) {
  for (int n = 0; n < num; ++n) {
    const uvlm_kinematics& k = kins[n];
    const double om[4] = {k.plug_omega, k.flap_omega, k.twist_omega, k.bend_omega};
    double w = 0;
    for (double o : om)
      if (o != 0.0) {
        w = o;
        break;
      }
    h_phase[n] = w * t;
  }
  UVLM_CUDA_TRY(cudaMemcpyAsync(d_phase, h_phase, sizeof(double) * num, cudaMemcpyHostToDevice, st));
  return ok();
}

Error uvlm_ctx::warm_features(double t) {
  UVLM_TRY(warm_phase(t));
  return mlp_features(num, R, C, d_gamma_prev, d_gamma_hist, d_rhs, d_rhs_prev, d_phase, d_feat, st);
}

Error uvlm_ctx::step(long long step, double dt, double* row) {
  UVLM_TRY(stage_kinematics(step, dt));
  UVLM_TRY(stage_assemble());
  UVLM_TRY(stage_rhs());
  UVLM_TRY(stage_solve());
  UVLM_TRY(stage_loads());
  return stage_advect(row);
}

// Wing motion, shed, collocation points and normals (simple_simulator.cpp:241-262).
Error uvlm_ctx::stage_kinematics(long long step, double dt) {
  if (!built) return fail(kErrState, "uvlm_begin has not been called");
  const double t = step * dt;
  stage_step = step;
  cur_dt = dt;
  work_nbody = work_asm = work_lu = 0;
  nbev_n = 0;
  fev_used = false;
  last.initial_residual = 0;
  mark(0);
  UVLM_CUDA_TRY(cudaMemsetAsync(d_flags, 0, sizeof(int) * 4, st));
  UVLM_CUDA_TRY(cudaMemcpyAsync(d_gamma_hist, d_gamma_prev, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
  UVLM_CUDA_TRY(cudaMemcpyAsync(d_gamma_prev, d_gamma, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
  UVLM_TRY(launch_kinematics(d_kin, ws(), d_pos_init, d_pos, t, st));
  if (wake_nodes + 1 > PR) return fail(kErrCapacity, "wake longer than max_wake_rows");
  UVLM_TRY(shed(step));
  UVLM_TRY(launch_panel_geometry(d_kin, ws(), d_pos, d_pos_init, t, d_cx, d_cy, d_cz, d_normal, d_area, d_uls, st));
  mark(1);
  return ok();
}

Error uvlm_ctx::stage_assemble() {
  // influence matrix (simple_simulator.cpp:76-101)
  // Mixed form: the matrix of the FP64 residual is assembled every step, in
  // FP64 (assembly_fp64) or by the FP32 kernel; the FP32 matrix that is
  // factored is assembled by the FP32 kernel only when a factorisation runs.
  if (mixed()) {
    if (cfg.assembly_fp64)
      UVLM_TRY(launch_assemble(ws(), d_pos, d_cx, d_cy, d_cz, d_normal, false, d_A64, false, st));
    else
      UVLM_TRY(launch_assemble(ws(), d_pos, d_cx, d_cy, d_cz, d_normal, true, d_A32, true, st));
  } else {
    UVLM_TRY(launch_assemble(ws(), d_pos, d_cx, d_cy, d_cz, d_normal, false, d_A64, false, st));
  }
  work_asm = (double)N * (double)N * 4.0;
  mark(2);
  return ok();
}

Error uvlm_ctx::stage_rhs() {
  // RHS: wake normal wash at the collocation points (:103-124)
  {
    SourceBlock blocks[2];
    int nbk = 0;
    const NBodyPrec prec = stage_prec(UVLM_STAGE_RHS);
    nb.near64 = stage_near64(UVLM_STAGE_RHS);
    UVLM_TRY(build_sources(false, d_wpos, prec, blocks, &nbk));
    UVLM_CUDA_TRY(cudaMemcpyAsync(d_tx, d_cx, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    UVLM_CUDA_TRY(cudaMemcpyAsync(d_ty, d_cy, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    UVLM_CUDA_TRY(cudaMemcpyAsync(d_tz, d_cz, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    UVLM_TRY(eval(blocks, nbk, N, prec, kStageRhs));
    UVLM_TRY(launch_rhs(N, d_vx, d_vy, d_vz, d_uls, d_normal, ff, d_rhs, st));
  }
  mark(3);
  return ok();
}

Error uvlm_ctx::stage_solve() {
  const long long step = stage_step;
  const double t = step * cur_dt;
  UVLM_TRY(solve(step));
  UVLM_TRY(launch_check_finite(d_gamma, N, d_flags, st));
  if (collect && step >= 2 && collect_n + N <= collect_cap) {
    // training pair of the learned warm start: features known before the
    // solve, target = the solved circulation minus the extrapolation
    UVLM_TRY(warm_features(t));
    UVLM_CUDA_TRY(cudaMemcpyAsync(d_collect_x + collect_n * kMlpIn, d_feat, sizeof(float) * N * kMlpIn,
                                  cudaMemcpyDeviceToDevice, st));
    UVLM_TRY(mlp_targets(N, d_gamma, d_gamma_prev, d_gamma_hist, d_collect_t + collect_n, st));
    collect_n += N;
  }
  UVLM_CUDA_TRY(cudaMemcpyAsync(d_rhs_prev, d_rhs, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
  if (out)  // OutputPanels / OutputSheet after the solve (simple_simulator.cpp:270-277)
    UVLM_TRY(output_enqueue(out, OutputState{num, R, C, PR, wake_start, wake_nodes, d_pos, d_gamma, d_wpos, d_wgamma},
                            t, st));
  mark(4);
  return ok();
}

Error uvlm_ctx::stage_loads() {
  const double t = stage_step * cur_dt, dt = cur_dt;
  if (cfg.compute_loads) {
    const long long lines = (long long)num * R * (2 * C + 1);
    UVLM_TRY(launch_line_prep(d_kin, ws(), d_pos, d_pos_init, t, d_tx, d_ty, d_tz, d_line_uls, st));
    SourceBlock blocks[2];
    int nbk = 0;
    const NBodyPrec prec = stage_prec(UVLM_STAGE_LOADS);
    nb.near64 = stage_near64(UVLM_STAGE_LOADS);
    UVLM_TRY(build_sources(true, d_wpos, prec, blocks, &nbk));
    UVLM_TRY(eval(blocks, nbk, lines, prec, kStageLoads));
    UVLM_TRY(launch_loads(ws(), d_pos, d_gamma, d_gamma_prev, d_normal, d_area, d_vx, d_vy, d_vz, d_line_uls, ff,
                          d_chord_span, t, dt, d_row, st));
  }
  mark(5);
  return ok();
}

// Advect (:284), the erase of the oldest wake row, and the end of the step:
// the load row and the error words back to the host.
Error uvlm_ctx::stage_advect(double* row) {
  const long long step = stage_step;
  const double dt = cur_dt, t = step * dt;
  UVLM_TRY(advect(dt));
  mark(6);
  if (cfg.erase_wake_after > 0 && step >= cfg.erase_wake_after && wake_nodes > 0) wake_nodes -= 1;
  // end of step: load row and error words back to the host
  UVLM_CUDA_TRY(cudaMemcpyAsync(h_row, d_row, sizeof(double) * (1 + 2 * num), cudaMemcpyDeviceToHost, st));
  UVLM_CUDA_TRY(cudaMemcpyAsync(h_flags, d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
  UVLM_CUDA_TRY(cudaMemcpyAsync(h_flags + 4, lu.err, sizeof(int) * 4, cudaMemcpyDeviceToHost, st));
  h_flags[8] = 0;
  Mlp* tcm = mlp_tc_used && mlp ? mlp_of(mlp) : nullptr;
  if (tcm && tcm->tc_err)
    UVLM_CUDA_TRY(cudaMemcpyAsync(h_flags + 8, tcm->tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  mlp_tc_used = false;
  mark(7);
  UVLM_CUDA_TRY(cudaStreamSynchronize(st));
  if (h_flags[4]) return fail(kErrTimeout, "a bounded device wait in the dense solve gave up");
  if (h_flags[8]) {
    UVLM_CUDA_TRY(cudaMemset(tcm->tc_err, 0, sizeof(int)));
    return fail(kErrTimeout, "a bounded device wait of the tensor-core warm start gave up");
  }
  if (h_flags[5]) return fail(kErrSingular, "zero pivot in the LU factorisation");
  if (h_flags[0]) return fail(kErrNonFinite, "non-finite circulation after the solve");
  if (!cfg.compute_loads) {
    h_row[0] = t;
    for (int i = 1; i < 1 + 2 * num; ++i) h_row[i] = 0;
  }
  if (row) std::memcpy(row, h_row, sizeof(double) * (1 + 2 * num));
  last.step = step;
  last.t = t;
  last.wake_rows = wake_rings();
  {
    const int pm = mixed() ? 0 : 1;
    last.nbody_variant = stage_variant[kStageAdvect][pm];
    last.stage_variant[0] = stage_variant[kStageRhs][stage_prec(UVLM_STAGE_RHS) == kNBodyFP64 ? 1 : 0];
    last.stage_variant[1] = stage_variant[kStageLoads][stage_prec(UVLM_STAGE_LOADS) == kNBodyFP64 ? 1 : 0];
    last.stage_variant[2] = stage_variant[kStageAdvect][stage_prec(UVLM_STAGE_ADVECT) == kNBodyFP64 ? 1 : 0];
    last.stage_variant[3] = -1;
    (void)pm;
  }
  if (timing) {
    float ms[8] = {0};
    const int map[7][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {0, 7}};
    for (int q = 0; q < 7; ++q) cudaEventElapsedTime(&ms[q], ev[map[q][0]], ev[map[q][1]]);
    last.stage_ms[0] = ms[0];
    last.stage_ms[1] = ms[1];
    last.stage_ms[2] = ms[2];
    last.stage_ms[3] = ms[3];
    last.stage_ms[4] = ms[4];
    last.stage_ms[5] = ms[5];
    last.stage_ms[6] = 0;
    last.stage_ms[7] = ms[6];
    double nbt = 0;
    for (int q = 0; q < nbev_n; ++q) {
      float m = 0;
      cudaEventElapsedTime(&m, nbev[2 * q], nbev[2 * q + 1]);
      nbt += m;
    }
    last.nbody_ms = nbt;
    last.factor_ms = last.inverse_ms = 0;
    if (fev_used) {
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, fev[0], fev[1]);
      cudaEventElapsedTime(&b, fev[1], fev[2]);
      last.factor_ms = a;
      last.inverse_ms = b;
    }
  }
  nbev_n = 0;
  return ok();
}

// =================================================================== C-ABI
extern "C" {

void uvlm_config_default(uvlm_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->precision = UVLM_PRECISION_FP64;
  c->solver = UVLM_SOLVER_LU;
  c->warm_start = UVLM_WARM_PREVIOUS;
  c->lu_precision = UVLM_LU_TF32;
  // mixed form: the RHS stage's near pairs in FP64 (the wake's newest rows sit
  // next to the trailing-edge collocation points; their FP32 rounding is the
  // largest source of circulation error, for 0.2 % of the step's time)
  c->nbody_near_fp64 = UVLM_STAGE_RHS;
  c->advection = UVLM_ADVECT_EULER;
  c->rk_ignore_rows = 5;
  c->max_wake_rows = 1024;
  c->erase_wake_after = 0;
  c->gmres_restart = 20;
  c->gmres_max_iter = 20;
  c->gmres_tol = 1e-12;
  c->device = 0;
  c->compute_loads = 1;
  c->assembly_fp64 = 0;
  c->nbody_variant = -1;
  c->preconditioner = UVLM_PRECOND_INVERSE;
  // the preconditioner's pivots among each panel's top 256 rows: on the
  // influence matrices of the path the largest entry of every column lies
  // there, so the factors (and every GMRES iterate) are the same as with the
  // panel-wide tournament, for 0.65x the factorisation time
  c->lu_pivoting = UVLM_PIVOT_LOCAL;
  c->gmres_refresh_iter = 16;
}

const char* uvlm_status_string(int s) {
  switch (s) {
    case UVLM_OK: return "ok";
    case UVLM_ERR_INVALID: return "invalid argument";
    case UVLM_ERR_CUDA: return "CUDA error";
    case UVLM_ERR_SINGULAR: return "singular matrix";
    case UVLM_ERR_NONFINITE: return "non-finite value";
    case UVLM_ERR_STATE: return "call out of order";
    case UVLM_ERR_CAPACITY: return "capacity exceeded";
    case UVLM_ERR_TIMEOUT: return "device wait timed out";
    case UVLM_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

const char* uvlm_global_last_error(void) { return g_last_error.c_str(); }

int uvlm_create(const uvlm_config* cfg, uvlm_ctx** out) {
  if (!out) return set_global(fail(kErrInvalid, "out is NULL"));
  *out = nullptr;
  uvlm_ctx* c = new uvlm_ctx();
  if (cfg)
    c->cfg = *cfg;
  else
    uvlm_config_default(&c->cfg);
  const uvlm_config& k = c->cfg;
  if (k.precision != UVLM_PRECISION_FP64 && k.precision != UVLM_PRECISION_MIXED) {
    delete c;
    return set_global(fail(kErrInvalid, "unknown precision"));
  }
  if (k.advection < 0 || k.advection > 3 || k.max_wake_rows < 1 || k.gmres_restart < 1 || k.gmres_max_iter < 1 ||
      !(k.gmres_tol > 0) || k.preconditioner < 0 || k.preconditioner > 1 || k.nbody_fp64_stages < 0 ||
      k.nbody_fp64_stages > (UVLM_STAGE_RHS | UVLM_STAGE_LOADS | UVLM_STAGE_ADVECT) || k.nbody_near_fp64 < 0 ||
      k.nbody_near_fp64 > (UVLM_STAGE_RHS | UVLM_STAGE_LOADS | UVLM_STAGE_ADVECT) ||
      (k.lu_pivoting != UVLM_PIVOT_PANEL && k.lu_pivoting != UVLM_PIVOT_LOCAL) || k.gmres_refresh_iter < 0) {
    delete c;
    return set_global(fail(kErrInvalid, "invalid configuration"));
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    delete c;
    cudaGetLastError();
    return set_global(fail(kErrCuda, "no CUDA device"));
  }
  if (cudaSetDevice(k.device) != cudaSuccess) {
    delete c;
    return set_global(fail(kErrCuda, "cudaSetDevice failed"));
  }
  c->num_sms = device_sms(k.device);
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return set_global(fail(kErrCuda, "cudaStreamCreate failed"));
  }
  for (auto& e : c->ev) cudaEventCreate(&e);
  for (auto& e : c->nbev) cudaEventCreate(&e);
  for (auto& e : c->fev) cudaEventCreate(&e);
  if (k.nbody_variant >= 0) {
    if (k.nbody_variant >= nbody_num_variants()) {
      uvlm_destroy(c);
      return set_global(fail(kErrInvalid, "nbody_variant out of range"));
    }
    if (k.precision == UVLM_PRECISION_MIXED && k.nbody_near_fp64 && !nbody_variant_near64(k.nbody_variant)) {
      uvlm_destroy(c);
      return set_global(fail(kErrInvalid, "nbody_near_fp64 needs a packed far-field FP32 tile (\"fp32_*_t2_*_x2f\")"));
    }
    // the pinned tile serves every stage of its precision
    const int pi = nbody_variant_prec(k.nbody_variant) == kNBodyFP64 ? 1 : 0;
    for (int st = 0; st < 3; ++st) {
      c->stage_variant[st][pi] = k.nbody_variant;
      c->stage_pinned[st][pi] = true;
    }
  }
  *out = c;
  return UVLM_OK;
}

int uvlm_destroy(uvlm_ctx* c) {
  if (!c) return UVLM_OK;
  if (c->st) cudaStreamSynchronize(c->st);
  const Error oe = output_close(c->out);
  c->out = nullptr;
  c->free_all();
  cudaFree(c->d_collect_x);
  cudaFree(c->d_collect_t);
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->nbev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c->fev)
    if (e) cudaEventDestroy(e);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return oe.code ? set_global(oe) : UVLM_OK;
}

int uvlm_set_output_paths(uvlm_ctx* c, const char* sheet_path, const char* result_path) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (c->st) cudaStreamSynchronize(c->st);
  Error e = output_close(c->out);
  c->out = nullptr;
  if (e.code) return c->fail_with(e);
  if ((sheet_path && *sheet_path) || (result_path && *result_path))
    e = output_open(&c->out, sheet_path, result_path, c->cfg.device);
  return c->fail_with(e);
}

int uvlm_flush_output(uvlm_ctx* c) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (!c->out) return UVLM_OK;
  if (c->st) cudaStreamSynchronize(c->st);
  return c->fail_with(output_flush(c->out));
}

int uvlm_write_state_record(const char* path, int32_t append, int32_t kind, int64_t num, int64_t rows, int64_t cols,
                            int64_t wake_rows, const double* wing_pos, const double* wing_gamma,
                            const double* wake_pos, const double* wake_gamma, double t) {
  if (!path || (kind != UVLM_OUTPUT_SHEETS && kind != UVLM_OUTPUT_SNAPSHOT2) || num < 0 || rows < 0 || cols < 0 ||
      wake_rows < 0 || !wing_pos || !wake_pos || (num * rows * cols > 0 && !wing_gamma) ||
      (num * wake_rows * cols > 0 && !wake_gamma))
    return set_global(fail(kErrInvalid, "invalid argument"));
  return set_global(output_encode_to_file(path, append, kind, (int)num, (int)rows, (int)cols, (int)wake_rows, wing_pos,
                                          wing_gamma, wake_pos, wake_gamma, t));
}

int uvlm_write_legacy_snapshot2(const char* path, double t, int64_t n_containers, const int64_t* rows,
                                const int64_t* cols, const double* chord, const double* span, const double* rings,
                                const double* rings0, const double* gamma, int64_t n_rings, const double* mv_center,
                                const double* mv_nodes, const double* mv_freestream, int64_t n_mv) {
  if (!path || n_containers < 0 || n_rings < 0 || n_mv < 0 ||
      (n_containers > 0 && (!rows || !cols || !chord || !span)) || (n_rings > 0 && (!rings || !gamma)) ||
      (n_mv > 0 && (!mv_center || !mv_nodes || !mv_freestream)))
    return set_global(fail(kErrInvalid, "invalid argument"));
  for (int64_t c = 0; c < n_containers; ++c)
    if (rows[c] < 0 || cols[c] < 0 || rows[c] > 0xFFFFFFFFll || cols[c] > 0xFFFFFFFFll)
      return set_global(fail(kErrInvalid, "container shape out of range"));
  const LegacySnapshot s{n_containers, rows,  cols,  chord, span,     n_rings,      rings,
                         rings0,       gamma, n_mv, mv_center, mv_nodes, mv_freestream};
  return set_global(output_write_legacy_snapshot2(path, t, s));
}

const char* uvlm_last_error(const uvlm_ctx* c) { return c ? c->err.c_str() : g_last_error.c_str(); }

int uvlm_add_wing(uvlm_ctx* c, const uvlm_wing_desc* w, const uvlm_kinematics* kin) {
  if (!c || !w) return set_global(fail(kErrInvalid, "NULL argument"));
  if (c->built) return c->fail_with(fail(kErrState, "wings are added before uvlm_begin"));
  if (w->rows < 1 || w->cols < 2 || (w->cols & 1) || !(w->chord > 0) || !(w->span > 0))
    return c->fail_with(fail(kErrInvalid, "rows >= 1, even cols >= 2 and positive chord/span are required"));
  if (!c->wings.empty() && (c->wings.back().rows != w->rows || c->wings.back().cols != w->cols))
    return c->fail_with(fail(kErrInvalid, "all wings must have the same rows and cols"));
  c->wings.push_back(*w);
  c->wing_nodes.emplace_back();
  uvlm_kinematics k{};
  if (kin) k = *kin;
  // BuildWing sets the morphing origin to the wing origin (simple_simulator.cpp:157)
  for (int d = 0; d < 3; ++d) k.origin[d] = w->origin[d];
  c->kins.push_back(k);
  return UVLM_OK;
}

int uvlm_add_wing_nodes(uvlm_ctx* c, int64_t rows, int64_t cols, const double* nodes, double chord, double span,
                        const double origin[3], const uvlm_kinematics* kin) {
  if (!c || !nodes || !origin) return set_global(fail(kErrInvalid, "NULL argument"));
  if (c->built) return c->fail_with(fail(kErrState, "wings are added before uvlm_begin"));
  if (rows < 1 || cols < 1 || rows > (1 << 20) || cols > (1 << 20) || !(chord > 0) || !(span > 0))
    return c->fail_with(fail(kErrInvalid, "rows >= 1, cols >= 1 and positive chord/span are required"));
  if (!c->wings.empty() && (c->wings.back().rows != rows || c->wings.back().cols != cols))
    return c->fail_with(fail(kErrInvalid, "all wings must have the same rows and cols"));
  const size_t cnt = (size_t)(rows + 1) * (size_t)(cols + 1) * 3;
  for (size_t q = 0; q < cnt; ++q)
    if (!std::isfinite(nodes[q])) return c->fail_with(fail(kErrInvalid, "non-finite wing node"));
  uvlm_wing_desc w{};
  w.chord = chord;
  w.span = span;
  w.rows = rows;
  w.cols = cols;
  for (int d = 0; d < 3; ++d) w.origin[d] = origin[d];
  c->wings.push_back(w);
  c->wing_nodes.emplace_back(nodes, nodes + cnt);
  uvlm_kinematics k{};
  if (kin) k = *kin;
  for (int d = 0; d < 3; ++d) k.origin[d] = origin[d];
  c->kins.push_back(k);
  return UVLM_OK;
}

int uvlm_set_forward_flight(uvlm_ctx* c, const double ff[3]) {
  if (!c || !ff) return set_global(fail(kErrInvalid, "NULL argument"));
  for (int d = 0; d < 3; ++d) c->ff[d] = ff[d];
  return UVLM_OK;
}

int uvlm_set_advection(uvlm_ctx* c, const char* name) {
  if (!c || !name) return set_global(fail(kErrInvalid, "NULL argument"));
  const std::string s(name);
  int a = -1;
  if (s == "euler") a = UVLM_ADVECT_EULER;
  if (s == "RK2") a = UVLM_ADVECT_RK2;
  if (s == "RK4") a = UVLM_ADVECT_RK4;
  if (s == "AB2") a = UVLM_ADVECT_AB2;
  if (a < 0) return c->fail_with(fail(kErrInvalid, "Invalid advection name! Please choose from following: [AB2, RK2, RK4, euler]"));
  c->cfg.advection = a;
  c->has_vprev = false;
  return UVLM_OK;
}

int uvlm_begin(uvlm_ctx* c) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (c->wings.empty()) return c->fail_with(fail(kErrState, "call uvlm_add_wing at least once"));
  cudaSetDevice(c->cfg.device);
  c->stage_next = 0;
  c->num = (int)c->wings.size();
  c->R = (int)c->wings[0].rows;
  c->C = (int)c->wings[0].cols;
  c->N = c->num * c->R * c->C;
  c->PR = (int)c->cfg.max_wake_rows + 2 + 64;
  Error e = c->alloc_all();
  if (e.code) return c->fail_with(e);
  std::vector<double> nodes;
  for (size_t q = 0; q < c->wings.size(); ++q) {
    const auto& w = c->wings[q];
    if (c->wing_nodes[q].empty()) {
      auto v = whole_wing_nodes(w);
      nodes.insert(nodes.end(), v.begin(), v.end());
    } else {
      // the caller's lattice (points of WholeWing) moved to the wing origin
      // (simple_simulator.cpp:162-166)
      const auto& v = c->wing_nodes[q];
      for (size_t k = 0; k < v.size(); ++k) nodes.push_back(v[k] + w.origin[k % 3]);
    }
  }
  if (cudaMemcpy(c->d_pos_init, nodes.data(), sizeof(double) * nodes.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_pos, nodes.data(), sizeof(double) * nodes.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_kin, c->kins.data(), sizeof(uvlm_kinematics) * c->kins.size(), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemset(c->d_gamma, 0, sizeof(double) * c->N) != cudaSuccess ||
      cudaMemset(c->d_gamma_prev, 0, sizeof(double) * c->N) != cudaSuccess ||
      cudaMemset(c->d_row, 0, sizeof(double) * (1 + 2 * c->num)) != cudaSuccess)
    return c->fail_with(fail(kErrCuda, "initial upload failed"));
  c->wake_start = c->PR;
  c->wake_nodes = 0;
  c->has_vprev = false;
  c->have_factors = false;
  c->built = true;
  return UVLM_OK;
}

int uvlm_step(uvlm_ctx* c, int64_t step, double dt, double* row) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (!(dt > 0)) return c->fail_with(fail(kErrInvalid, "dt must be positive"));
  if (c->stage_next) return c->fail_with(fail(kErrState, "a staged MainLoop is in progress"));
  return c->fail_with(c->step(step, dt, row));
}

// The staged MainLoop: each call checks that it is the stage expected next;
// an error abandons the step (the next call must be uvlm_stage_kinematics).
static int run_stage(uvlm_ctx* c, int stage, const std::function<Error()>& fn) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (c->stage_next != stage) {
    static const char* names[] = {"uvlm_stage_kinematics", "uvlm_stage_assemble", "uvlm_stage_rhs",
                                  "uvlm_stage_solve",      "uvlm_stage_loads",    "uvlm_stage_advect"};
    return c->fail_with(fail(kErrState, std::string("stage out of order: expected ") + names[c->stage_next]));
  }
  const Error e = fn();
  c->stage_next = e.code ? 0 : (stage + 1) % 6;
  return c->fail_with(e);
}

int uvlm_stage_kinematics(uvlm_ctx* c, int64_t step, double dt) {
  if (c && !(dt > 0)) return c->fail_with(fail(kErrInvalid, "dt must be positive"));
  return run_stage(c, 0, [&] { return c->stage_kinematics(step, dt); });
}
int uvlm_stage_assemble(uvlm_ctx* c) { return run_stage(c, 1, [&] { return c->stage_assemble(); }); }
int uvlm_stage_rhs(uvlm_ctx* c) { return run_stage(c, 2, [&] { return c->stage_rhs(); }); }
int uvlm_stage_solve(uvlm_ctx* c) { return run_stage(c, 3, [&] { return c->stage_solve(); }); }
int uvlm_stage_loads(uvlm_ctx* c) { return run_stage(c, 4, [&] { return c->stage_loads(); }); }
int uvlm_stage_advect(uvlm_ctx* c, double* row) { return run_stage(c, 5, [&] { return c->stage_advect(row); }); }

int uvlm_run(uvlm_ctx* c, int64_t steps, double dt, double* loads) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  int rc = uvlm_begin(c);
  if (rc) return rc;
  for (int64_t s = 0; s <= steps; ++s) {
    rc = uvlm_step(c, s, dt, loads ? loads + s * (1 + 2 * c->num) : nullptr);
    if (rc) return rc;
  }
  return UVLM_OK;
}

int uvlm_erase_oldest_wake(uvlm_ctx* c) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (!c->built) return c->fail_with(fail(kErrState, "uvlm_begin has not been called"));
  if (c->stage_next) return c->fail_with(fail(kErrState, "a staged MainLoop is in progress"));
  if (c->wake_nodes > 0) c->wake_nodes -= 1;
  return UVLM_OK;
}

int uvlm_get_sizes(const uvlm_ctx* c, int64_t* num, int64_t* rows, int64_t* cols, int64_t* wake_rows,
                   int64_t* wake_node_rows) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (num) *num = c->built ? c->num : (int64_t)c->wings.size();
  if (rows) *rows = c->built ? c->R : (c->wings.empty() ? 0 : c->wings[0].rows);
  if (cols) *cols = c->built ? c->C : (c->wings.empty() ? 0 : c->wings[0].cols);
  if (wake_rows) *wake_rows = c->wake_rings();
  if (wake_node_rows) *wake_node_rows = c->wake_nodes;
  return UVLM_OK;
}

static Error copy_wake_out(uvlm_ctx* c, const double* src, double* dst, int row_elems, int rows) {
  for (int n = 0; n < c->num; ++n) {
    const double* s = src + ((size_t)n * c->PR + c->wake_start) * row_elems;
    UVLM_CUDA_TRY(cudaMemcpy(dst + (size_t)n * rows * row_elems, s, sizeof(double) * rows * row_elems,
                             cudaMemcpyDeviceToHost));
  }
  return ok();
}

int uvlm_get_state(uvlm_ctx* c, double* wing_pos, double* wing_pos_init, double* wake_pos, double* wing_gamma,
                   double* wing_gamma_prev, double* wake_gamma) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (!c->built) return c->fail_with(fail(kErrState, "uvlm_begin has not been called"));
  if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->fail_with(fail(kErrCuda, "stream sync failed"));
  const size_t nn = (size_t)c->num * (c->R + 1) * (c->C + 1) * 3;
  Error e;
  auto cp = [&](double* dst, const double* src, size_t cnt) {
    if (dst && !e.code && cudaMemcpy(dst, src, sizeof(double) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess)
      e = fail(kErrCuda, "state copy failed");
  };
  cp(wing_pos, c->d_pos, nn);
  cp(wing_pos_init, c->d_pos_init, nn);
  cp(wing_gamma, c->d_gamma, (size_t)c->N);
  cp(wing_gamma_prev, c->d_gamma_prev, (size_t)c->N);
  if (!e.code && wake_pos && c->wake_nodes > 0) e = copy_wake_out(c, c->d_wpos, wake_pos, 3 * (c->C + 1), c->wake_nodes);
  if (!e.code && wake_gamma && c->wake_rings() > 0) e = copy_wake_out(c, c->d_wgamma, wake_gamma, c->C, c->wake_rings());
  return c->fail_with(e);
}

int uvlm_set_state(uvlm_ctx* c, int64_t wake_rows, const double* wing_pos, const double* wake_pos,
                   const double* wing_gamma, const double* wing_gamma_prev, const double* wake_gamma) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (!c->built) return c->fail_with(fail(kErrState, "uvlm_begin has not been called"));
  if (c->stage_next) return c->fail_with(fail(kErrState, "a staged MainLoop is in progress"));
  if (wake_rows < 0 || wake_rows + 2 > c->PR) return c->fail_with(fail(kErrCapacity, "wake_rows exceeds capacity"));
  if (!wing_pos || !wake_pos || !wing_gamma || !wing_gamma_prev || (wake_rows > 0 && !wake_gamma))
    return c->fail_with(fail(kErrInvalid, "NULL state array"));
  cudaStreamSynchronize(c->st);
  const size_t nn = (size_t)c->num * (c->R + 1) * (c->C + 1) * 3;
  const int nodes = (int)wake_rows + 1;
  c->wake_start = c->PR - nodes - 1;
  c->wake_nodes = nodes;
  Error e;
  auto up = [&](double* dst, const double* src, size_t cnt) {
    if (!e.code && cudaMemcpy(dst, src, sizeof(double) * cnt, cudaMemcpyHostToDevice) != cudaSuccess)
      e = fail(kErrCuda, "state upload failed");
  };
  up(c->d_pos, wing_pos, nn);
  up(c->d_gamma, wing_gamma, (size_t)c->N);
  up(c->d_gamma_prev, wing_gamma_prev, (size_t)c->N);
  for (int n = 0; n < c->num && !e.code; ++n) {
    up(c->d_wpos + ((size_t)n * c->PR + c->wake_start) * 3 * (c->C + 1), wake_pos + (size_t)n * nodes * 3 * (c->C + 1),
       (size_t)nodes * 3 * (c->C + 1));
    if (wake_rows > 0)
      up(c->d_wgamma + ((size_t)n * c->PR + c->wake_start) * c->C, wake_gamma + (size_t)n * wake_rows * c->C,
         (size_t)wake_rows * c->C);
  }
  c->has_vprev = false;
  c->have_factors = false;
  return c->fail_with(e);
}

int uvlm_get_last_stats(const uvlm_ctx* c, uvlm_step_stats* s) {
  if (!c || !s) return set_global(fail(kErrInvalid, "NULL argument"));
  *s = c->last;
  return UVLM_OK;
}

int uvlm_set_stage_timing(uvlm_ctx* c, int32_t enable) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  c->timing = enable != 0;
  return UVLM_OK;
}

int uvlm_synchronize(uvlm_ctx* c) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (cudaStreamSynchronize(c->st) != cudaSuccess) return c->fail_with(fail(kErrCuda, "stream sync failed"));
  return UVLM_OK;
}

void* uvlm_stream(uvlm_ctx* c) { return c ? (void*)c->st : nullptr; }

int64_t uvlm_kernel_launch_count(void) { return g_launches.load(); }

const char* uvlm_nbody_variant_name(int32_t v) { return nbody_variant_name(v); }

int uvlm_set_mlp(uvlm_ctx* c, uvlm_mlp* m) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  c->mlp = m;
  return UVLM_OK;
}

int uvlm_collect_training_data(uvlm_ctx* c, int32_t enable, int64_t max_samples) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  cudaFree(c->d_collect_x);
  cudaFree(c->d_collect_t);
  c->d_collect_x = nullptr;
  c->d_collect_t = nullptr;
  c->collect = false;
  c->collect_n = c->collect_cap = 0;
  if (!enable) return UVLM_OK;
  if (max_samples < 1) return c->fail_with(fail(kErrInvalid, "max_samples must be positive"));
  if (cudaMalloc(&c->d_collect_x, sizeof(float) * max_samples * kMlpIn) != cudaSuccess ||
      cudaMalloc(&c->d_collect_t, sizeof(float) * max_samples) != cudaSuccess)
    return c->fail_with(fail(kErrCuda, "cannot allocate the training-data buffer"));
  c->collect = true;
  c->collect_cap = max_samples;
  return UVLM_OK;
}

int uvlm_get_training_data(uvlm_ctx* c, float* X, float* T, int64_t* n) {
  if (!c || !n) return set_global(fail(kErrInvalid, "NULL argument"));
  *n = c->collect_n;
  if (c->collect_n == 0 || (!X && !T)) return UVLM_OK;
  cudaStreamSynchronize(c->st);
  if ((X && cudaMemcpy(X, c->d_collect_x, sizeof(float) * c->collect_n * kMlpIn, cudaMemcpyDeviceToHost) != cudaSuccess) ||
      (T && cudaMemcpy(T, c->d_collect_t, sizeof(float) * c->collect_n, cudaMemcpyDeviceToHost) != cudaSuccess))
    return c->fail_with(fail(kErrCuda, "training-data copy failed"));
  return UVLM_OK;
}

int uvlm_measure_fp32_peak(int32_t device, double* tflops) {
  if (!tflops) return set_global(fail(kErrInvalid, "NULL argument"));
  if (cudaSetDevice(device) != cudaSuccess) return set_global(fail(kErrCuda, "cudaSetDevice failed"));
  return set_global(measure_fp32_fma_peak(device_sms(device), tflops));
}

int uvlm_set_wait_limit(int32_t device, int64_t cycles) {
  if (cycles < 0) return set_global(fail(kErrInvalid, "negative wait limit"));
  if (cudaSetDevice(device) != cudaSuccess) return set_global(fail(kErrCuda, "cudaSetDevice failed"));
  Error e = lu_set_wait_limit((long long)cycles);
  if (!e.code) e = tc_set_wait_limit((long long)cycles);
  if (!e.code) e = mlp_tc_set_wait_limit((long long)cycles);
  return set_global(e);
}

int uvlm_check_bounded_wait(int32_t device, int64_t cycles) {
  if (cycles <= 0) return set_global(fail(kErrInvalid, "the wait limit must be positive"));
  if (cudaSetDevice(device) != cudaSuccess) return set_global(fail(kErrCuda, "cudaSetDevice failed"));
  bool gave_up = false;
  const Error e = lu_wait_probe((long long)cycles, &gave_up);
  if (e.code) return set_global(e);
  if (gave_up) return set_global(fail(kErrTimeout, "a bounded device wait gave up (as intended by the check)"));
  return UVLM_OK;
}

int uvlm_measure_fp64_peak(int32_t device, double* tflops) {
  if (!tflops) return set_global(fail(kErrInvalid, "NULL argument"));
  if (cudaSetDevice(device) != cudaSuccess) return set_global(fail(kErrCuda, "cudaSetDevice failed"));
  return set_global(measure_fp64_fma_peak(device_sms(device), tflops));
}

int uvlm_velocity_at(uvlm_ctx* c, const double* targets, int64_t n, int32_t include_freestream, double* out) {
  if (!c || (n > 0 && (!targets || !out)) || n < 0) return set_global(fail(kErrInvalid, "NULL argument"));
  if (!c->built) return c->fail_with(fail(kErrState, "uvlm_begin has not been called"));
  if (n == 0) return UVLM_OK;
  cudaSetDevice(c->cfg.device);
  auto run = [&]() -> Error {
    SourceBlock blocks[2];
    int nbk = 0;
    const NBodyPrec prec = c->mixed() ? kNBodyFP32 : kNBodyFP64;
    c->nb.near64 = c->stage_near64(UVLM_STAGE_ADVECT);  // a query sees what the wake nodes see
    UVLM_TRY(c->build_sources(true, c->d_wpos, prec, blocks, &nbk));
    std::vector<double> sx, sy, sz;
    for (int64_t k0 = 0; k0 < n; k0 += c->tcap) {
      const long long cnt = std::min<long long>(c->tcap, n - k0);
      sx.resize(cnt);
      sy.resize(cnt);
      sz.resize(cnt);
      for (long long q = 0; q < cnt; ++q) {
        sx[q] = targets[3 * (k0 + q)];
        sy[q] = targets[3 * (k0 + q) + 1];
        sz[q] = targets[3 * (k0 + q) + 2];
      }
      UVLM_CUDA_TRY(cudaMemcpyAsync(c->d_tx, sx.data(), sizeof(double) * cnt, cudaMemcpyHostToDevice, c->st));
      UVLM_CUDA_TRY(cudaMemcpyAsync(c->d_ty, sy.data(), sizeof(double) * cnt, cudaMemcpyHostToDevice, c->st));
      UVLM_CUDA_TRY(cudaMemcpyAsync(c->d_tz, sz.data(), sizeof(double) * cnt, cudaMemcpyHostToDevice, c->st));
      UVLM_TRY(c->eval(blocks, nbk, cnt, prec, uvlm_ctx::kStageAdvect));
      UVLM_CUDA_TRY(cudaMemcpyAsync(sx.data(), c->d_vx, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->st));
      UVLM_CUDA_TRY(cudaMemcpyAsync(sy.data(), c->d_vy, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->st));
      UVLM_CUDA_TRY(cudaMemcpyAsync(sz.data(), c->d_vz, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->st));
      UVLM_CUDA_TRY(cudaStreamSynchronize(c->st));
      const double f = include_freestream ? 1.0 : 0.0;
      for (long long q = 0; q < cnt; ++q) {
        out[3 * (k0 + q)] = sx[q] - f * c->ff[0];
        out[3 * (k0 + q) + 1] = sy[q] - f * c->ff[1];
        out[3 * (k0 + q) + 2] = sz[q] - f * c->ff[2];
      }
    }
    return ok();
  };
  return c->fail_with(run());
}

int uvlm_get_last_work(const uvlm_ctx* c, double* nbody_pairs, double* assembly_pairs, double* lu_flops) {
  if (!c) return set_global(fail(kErrInvalid, "NULL context"));
  if (nbody_pairs) *nbody_pairs = c->work_nbody;
  if (assembly_pairs) *assembly_pairs = c->work_asm;
  if (lu_flops) *lu_flops = c->work_lu;
  return UVLM_OK;
}

}  // extern "C"
