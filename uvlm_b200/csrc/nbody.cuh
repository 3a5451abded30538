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
  float4 hv;  // h0.y, h0.z, |s0|^2, |h0|^2 (squared lengths of the FP32 segment vectors)
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
  // FP32 form: the near pairs in FP64 (packed tiles with the far-field test),
  // which needs the FP64 records of the same sheets as well
  bool near64 = false;
  void* records64 = nullptr;  // RecD array, same indices as records
  long long records64_cap = 0;
};

// ------------------------------------------------------------ record build
__device__ inline double sheet_ring_gamma(const SheetView& v, int n, int i, int j) {
  const int R = v.node_rows - 1;
  if (i < 0 || i >= R || j < 0 || j >= v.cols) return 0.0;
  return v.gamma[((long long)n * v.g_rows_alloc + v.g_row0 + i) * v.cols + j];
}

// Record k (sheet-major, row-major) of a sheet view: node position, the
// spanwise S(i,j) and chordwise H(i,j) strengths and segment vectors.
template <class Rec>
__device__ inline Rec build_record(const SheetView& v, long long k) {
  const double s = 1.0 / (4.0 * kPi);
  const int C1 = v.cols + 1;
  const int j = (int)(k % C1);
  const long long nr = k / C1;
  const int i = (int)(nr % v.node_rows);
  const int n = (int)(nr / v.node_rows);
  const double* p = v.pos + (((long long)n * v.rows_alloc + v.row0 + i) * C1 + j) * 3;
  const int R = v.node_rows - 1;
  const double gS = (j < v.cols) ? sheet_ring_gamma(v, n, i, j) - sheet_ring_gamma(v, n, i - 1, j) : 0.0;
  const double gH =
      (i < R && !v.spanwise_only) ? sheet_ring_gamma(v, n, i, j - 1) - sheet_ring_gamma(v, n, i, j) : 0.0;
  double s0[3] = {0, 0, 0}, h0[3] = {0, 0, 0};
  if (j < v.cols)
    for (int d = 0; d < 3; ++d) s0[d] = p[3 + d] - p[d];
  if (i < R)
    for (int d = 0; d < 3; ++d) h0[d] = p[3 * C1 + d] - p[d];
  Rec r;
  if constexpr (sizeof(Rec) == sizeof(RecF)) {
    const float hx = (float)p[0], hy = (float)p[1], hz = (float)p[2];
    r.hi = make_float4(hx, hy, hz, (float)(gS * s));
    r.lo = make_float4((float)(p[0] - (double)hx), (float)(p[1] - (double)hy), (float)(p[2] - (double)hz),
                       (float)(gH * s));
    const float sx = (float)s0[0], sy = (float)s0[1], sz = (float)s0[2];
    const float ex = (float)h0[0], ey = (float)h0[1], ez = (float)h0[2];
    r.sv = make_float4(sx, sy, sz, ex);
    r.hv = make_float4(ey, ez, (float)((double)sx * sx + (double)sy * sy + (double)sz * sz),
                       (float)((double)ex * ex + (double)ey * ey + (double)ez * ez));
  } else {
    r.a = make_double4(p[0], p[1], p[2], gS * s);
    r.b = make_double4(gH * s, s0[0], s0[1], s0[2]);
    r.c = make_double4(h0[0], h0[1], h0[2], 0.0);
  }
  return r;
}

// ---------------------------------------------------------- strip decode
struct StripInfo {
  long long first;  // record index of node (i0, j0)
  int row_stride;   // cols + 1
  int n_rows;       // owned node rows
  int nr;           // node rows loaded (n_rows + has_lower)
  int n_cols;       // node columns in the chunk
  bool last_h;      // owns the chordwise segments of its last column
};

// Source blocks of one evaluation cut into strips of H owned node rows x
// kStripCols segment columns (sheet-major, row groups, column chunks).
struct Blocks {
  SourceBlock b[4];
  int n;
  int strips_per_sheet[4];
  int chunks[4];
  long long strip_begin[5];
};

// Fills B from the blocks that carry segments; returns the strip count.
__host__ __device__ inline long long fill_blocks(Blocks& B, const SourceBlock* blocks, int n_blocks, int H) {
  B.n = 0;
  long long strips = 0;
  for (int i = 0; i < n_blocks && B.n < 4; ++i) {
    const SourceBlock& sb = blocks[i];
    if (sb.num <= 0 || sb.node_rows < 2 || sb.cols <= 0) continue;  // no rings -> no segments
    B.b[B.n] = sb;
    const int groups = (sb.node_rows + H - 1) / H;
    const int chunks = (sb.cols + kStripCols - 1) / kStripCols;
    B.chunks[B.n] = chunks;
    B.strips_per_sheet[B.n] = groups * chunks;
    B.strip_begin[B.n] = strips;
    strips += (long long)sb.num * groups * chunks;
    B.n++;
  }
  B.strip_begin[B.n] = strips;
  return strips;
}

template <int H>
__device__ inline StripInfo decode_strip(const Blocks& B, long long s) {
  int bi = 0;
  while (bi + 1 < B.n && s >= B.strip_begin[bi + 1]) ++bi;
  const SourceBlock& sb = B.b[bi];
  const long long local = s - B.strip_begin[bi];
  const int sps = B.strips_per_sheet[bi];
  const int chunks = B.chunks[bi];
  const int n = (int)(local / sps);
  const int rem = (int)(local % sps);
  const int g = rem / chunks, c = rem % chunks;
  StripInfo si;
  const int i0 = g * H, j0 = c * kStripCols;
  si.n_rows = min(H, sb.node_rows - i0);
  si.nr = si.n_rows + ((i0 + si.n_rows < sb.node_rows) ? 1 : 0);
  si.n_cols = min(kStripCols, sb.cols - j0) + 1;
  si.last_h = (j0 + si.n_cols - 1 == sb.cols);
  si.row_stride = sb.cols + 1;
  si.first = sb.rec_off + ((long long)n * sb.node_rows + i0) * (sb.cols + 1) + j0;
  return si;
}

// ------------------------------------------------------ batched evaluation
// Many independent problems in one persistent launch: problem c has its own
// source blocks (records already built) and targets [tgt_off, tgt_off+n_tgt)
// of the shared SoA target arrays; its velocities land at the same indices.
// Work items = (problem, target tile, source split) with at most
// kBatchStripsPerItem strips each; every CTA strides over the items, so the
// launch shape is fixed while the problem sizes change from step to step.
constexpr int kBatchStripsPerItem = 8;

struct NBodyBatchInput {
  SourceBlock blocks[2];
  int n_blocks;
  long long tgt_off, n_tgt;
};

struct NBodyBatchPlan {
  Blocks B;
  long long n_strips, tgt_off, n_tgt;
  long long tiles, splits, item_off, part_off, tgt_prefix;
};

// A problem whose sheets fill at least 3/4 of the staged strip columns is
// walked as whole padded strips by the packed FP32x2 walker (FP32 only); the
// others by the general walker.  FP32 evaluations therefore run as two
// persistent launches, one per class.
__host__ __device__ inline bool batch_input_padded(const NBodyBatchInput& x) {
  bool any = false;
  for (int i = 0; i < x.n_blocks; ++i) {
    const SourceBlock& b = x.blocks[i];
    if (b.num <= 0 || b.node_rows < 2 || b.cols <= 0) continue;
    const long long chunks = (b.cols + kStripCols - 1) / kStripCols;
    if (4 * (b.cols + chunks) < 3 * chunks * (kStripCols + 1)) return false;
    any = true;
  }
  return any;
}

// Strip height of the batched tile of a precision and class.
int nbody_batch_rows(NBodyPrec prec, bool padded);
// Upper bound of the partial-sum doubles for the given inputs (host copy).
long long nbody_batch_partial_doubles(NBodyPrec prec, const NBodyBatchInput* in, int n);
// Persistent grid sizes used by nbody_batch_eval on this device, and the
// FP32 tile (strip height) the batch runs: tiles[t] is the grid of tile t.
constexpr int kNumBatchTilesF = 3;
struct NBodyBatchGrids {
  int general = 0, padded = 0;
  int tiles[kNumBatchTilesF] = {0, 0, 0};
  int tile = 0;
};
const char* nbody_batch_tile_name(NBodyPrec prec, int tile);
NBodyBatchGrids nbody_batch_grids(NBodyPrec prec, int num_sms);

// d_in: n problems on the device.  Plans on the device (one CTA), evaluates
// with `grid` persistent CTAs and reduces the splits; d_plan holds n plans
// and d_totals 4 counters.  status[0] is set non-zero when the partial
// buffer is too small (nothing is evaluated then).
Error nbody_batch_eval(NBodyPrec prec, const NBodyBatchInput* d_in, int n, const double* tx, const double* ty,
                       const double* tz, double* vx, double* vy, double* vz, const void* records, double* partial,
                       long long partial_cap, NBodyBatchPlan* d_plan, long long* d_totals, int* status,
                       const NBodyBatchGrids& grids, cudaStream_t st);

int nbody_num_variants();
int nbody_variant_prec(int v);
// Whether a variant evaluates the FP32 form's near pairs in FP64 when NBodyWork::near64 is set.
bool nbody_variant_near64(int v);
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
