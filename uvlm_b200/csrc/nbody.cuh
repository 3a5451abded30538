// nbody.cuh -- all-pairs Biot-Savart induced velocity over vortex-ring sheets.
//
// Replaces the serial inner loop of UVLM::InducedVelocity (src/velocity.h:14-24)
// -> VORING (src/vortex.cpp:145-160) -> BiotSavartLaw (src/vortex.cpp:21-39)
// that every N-body stage of SimpleSimulator::MainLoop runs: the wake RHS
// (simple_simulator.cpp:103-124), the load-line velocities (:195-233) and the
// wake advection (src/advect.h:26-46, src/advect.cpp:11-217).
//
// Reformulation (same arithmetic, no approximation): a ring sheet of R x C
// rings with circulation G(i,j) is the superposition of its UNIQUE lattice
// segments, each carrying the difference of the circulations of the two rings
// that share it:
//   spanwise  S(i,j): p(i,j) -> p(i,j+1),  g = G(i,j)   - G(i-1,j)   i in 0..R
//   chordwise H(i,j): p(i,j) -> p(i+1,j),  g = G(i,j-1) - G(i,j)     j in 0..C
// (G = 0 outside the sheet).  Biot-Savart is linear in g and odd under a
// reversal of the segment, and the cut-off depends only on the geometry, so
// this equals the reference's 4-segments-per-ring sum up to rounding while
// doing about half of the segment evaluations.  Node quantities (x - p,
// 1/|x - p|) are shared by the segments meeting at that node.
//
// Data layout in HBM: per evaluation a "record" array holds, for every node of
// every source sheet, its position, the vectors s0 = p(i,j+1) - p(i,j) and
// h0 = p(i+1,j) - p(i,j) of the spanwise segment to its right and the
// chordwise segment below it (FP64 differences rounded once), and their
// strengths (pre-scaled by 1/4pi):
//   FP32 form (64 B): position as a hi/lo float pair (x = x_hi + x_lo), so that
//              x - p keeps near-FP64 accuracy for near pairs;
//   FP64 form (96 B).
// With the segment vector r0 at hand the cross product is d = r0 x r1
// (= r1 x r2 of src/vortex.cpp:24-28) without the cancellation of two long,
// nearly parallel vectors.  Sources are walked in "strips" of H owned node
// rows x up to kStripCols node columns, staged through shared memory by
// cp.async double buffering.
#pragma once

#include "common.cuh"

namespace uvlm {

constexpr int kStripCols = 64;  // segments per strip row (nodes = +1)

struct alignas(16) RecF {
  float4 hi;  // x_hi, y_hi, z_hi, gS/(4 pi)
  float4 lo;  // x_lo, y_lo, z_lo, gH/(4 pi)
  float4 sv;  // s0.x, s0.y, s0.z, h0.x
  float4 hv;  // h0.y, h0.z, 0, 0
};
struct alignas(16) RecD {
  double4 a;  // x, y, z, gS/(4 pi)
  double4 b;  // gH/(4 pi), s0.x, s0.y, s0.z
  double4 c;  // h0.x, h0.y, h0.z, 0
};

// One contiguous block of sheets in the record array: num sheets of
// node_rows x (cols+1) nodes, sheet-major, row-major inside a sheet.
struct SourceBlock {
  long long rec_off;
  int num, node_rows, cols;
};

// Physical description of a node sheet stored as AoS doubles [n][row][j][3]
// with `rows_alloc` rows per sheet and logical row i at physical row row0+i.
struct SheetView {
  const double* pos;
  int rows_alloc, row0;
  const double* gamma;  // [n][rows_alloc][cols] with the same physical rows
  int g_rows_alloc, g_row0;
  int num, node_rows, cols;  // cols = rings per row (C)
  int spanwise_only = 0;     // 1: chordwise strengths forced to zero
};

enum NBodyPrec { kNBodyFP64 = 0, kNBodyFP32 = 1 };

// Tile/launch configuration chosen by the autotuner.
struct NBodyTune {
  int variant = 0;  // index into the compiled kernel variants
};

struct NBodyWork {
  // scratch owned by the caller
  void* records = nullptr;  // RecF or RecD array
  long long records_cap = 0;
  double* partial = nullptr;  // [splits][3][targets]
  long long partial_cap = 0;  // doubles
  long long max_splits = 0;   // > 0: at most this many source splits (bounded scratch)
};

int nbody_num_variants();
int nbody_variant_prec(int v);
const char* nbody_variant_name(int v);

// Build the source records of `n_views` sheets into work.records (blocks are
// appended in order) and fill blocks[].  Returns total records.
Error nbody_build_sources(const SheetView* views, int n_views, NBodyPrec prec,
                          NBodyWork* work, SourceBlock* blocks,
                          cudaStream_t st);

// vel[t] (SoA vx,vy,vz, length n_targets) = sum over all sources of the
// induced velocity at target t (SoA tx,ty,tz FP64).  Overwrites vel.
Error nbody_eval(const SourceBlock* blocks, int n_blocks, NBodyPrec prec,
                 const double* tx, const double* ty, const double* tz,
                 long long n_targets, double* vx, double* vy, double* vz,
                 NBodyWork* work, int variant, int num_sms, cudaStream_t st);

// Algorithmic unique-segment count of a set of blocks (for the roofline).
long long nbody_unique_segments(const SourceBlock* blocks, int n_blocks);

}  // namespace uvlm
