// nbody.cu -- strip-tiled Biot-Savart N-body (FP32 hi/lo and FP64 forms).
#include <type_traits>

#include "device_once.h"
#include "nbody.cuh"

namespace uvlm {
namespace {

template <class Rec>
__global__ void build_records_kernel(SheetView v, Rec* out) {
  const long long total = (long long)v.num * v.node_rows * (v.cols + 1);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x)
    out[k] = build_record<Rec>(v, k);
}

// cp.async 16-byte staging of one strip into shared memory ([r][j] records)
template <class Rec>
__device__ inline void stage_strip(Rec* sm, const Rec* rec, const StripInfo& si) {
  constexpr int kChunks = sizeof(Rec) / 16;
  const int total = si.nr * si.n_cols * kChunks;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    const int part = q % kChunks;
    const int rj = q / kChunks;
    const int r = rj / si.n_cols, j = rj % si.n_cols;
    const char* src = reinterpret_cast<const char*>(rec + si.first + (long long)r * si.row_stride + j) + 16 * part;
    char* dst = reinterpret_cast<char*>(sm + rj) + 16 * part;
    const unsigned sdst = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst), "l"(src));
  }
  asm volatile("cp.async.commit_group;");
}

// Full-tile staging: always (H + 1) x (kStripCols + 1) records; entries past
// the strip's rows or columns are all-zero records (zero strengths, zero
// segment vectors), whose segments have d = 0 and are cut exactly like a
// degenerate segment, so they add +0 to every target.
template <class Rec, int H>
__device__ inline void stage_strip_padded(Rec* sm, const Rec* rec, const StripInfo& si) {
  constexpr int kChunks = sizeof(Rec) / 16;
  constexpr int kCols = kStripCols + 1;
  constexpr int total = (H + 1) * kCols * kChunks;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    const int part = q % kChunks;
    const int rj = q / kChunks;
    const int r = rj / kCols, j = rj % kCols;
    char* dst = reinterpret_cast<char*>(sm + rj) + 16 * part;
    if (r < si.nr && j < si.n_cols) {
      const char* src = reinterpret_cast<const char*>(rec + si.first + (long long)r * si.row_stride + j) + 16 * part;
      const unsigned sdst = (unsigned)__cvta_generic_to_shared(dst);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst), "l"(src));
    } else {
      *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  asm volatile("cp.async.commit_group;");
}

// Row-padded staging for the column-bounded walkers: records (r, j), j <
// n_cols, at row stride kStripCols + 1; rows past the strip's node rows are
// all-zero records (their segments have d = 0 and are cut); columns from
// n_cols on are not written and never read.
template <class Rec, int H>
__device__ inline void stage_strip_rows(Rec* sm, const Rec* rec, const StripInfo& si) {
  constexpr int kChunks = sizeof(Rec) / 16;
  const int total = (H + 1) * si.n_cols * kChunks;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    const int part = q % kChunks;
    const int rj = q / kChunks;
    const int r = rj / si.n_cols, j = rj % si.n_cols;
    char* dst = reinterpret_cast<char*>(sm + r * (kStripCols + 1) + j) + 16 * part;
    if (r < si.nr) {
      const char* src = reinterpret_cast<const char*>(rec + si.first + (long long)r * si.row_stride + j) + 16 * part;
      const unsigned sdst = (unsigned)__cvta_generic_to_shared(dst);
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sdst), "l"(src));
    } else {
      *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  asm volatile("cp.async.commit_group;");
}

template <class T>
struct Tgt {
  T hx, hy, hz;  // FP32: hi part; FP64: the position
  T lx, ly, lz;  // FP32: lo part; FP64: unused
};

template <class T>
struct NodeV {
  T rx, ry, rz;  // x - p
  T n;           // |x - p| (0 when x == p; such pairs are cut by |d|^2)
};

__device__ __forceinline__ float nb_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float nb_rcp(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <class T, class Rec>
__device__ __forceinline__ NodeV<T> node_from(const Rec& r, const Tgt<T>& t) {
  NodeV<T> n;
  if constexpr (sizeof(T) == 4) {
    n.rx = (t.hx - r.hi.x) + (t.lx - r.lo.x);
    n.ry = (t.hy - r.hi.y) + (t.ly - r.lo.y);
    n.rz = (t.hz - r.hi.z) + (t.lz - r.lo.z);
    const float q = n.rx * n.rx + n.ry * n.ry + n.rz * n.rz;
    n.n = q >= (float)kCutR2 ? q * nb_rsqrt(q) : 0.f;  // |x - p| < 1e-10: marked 0 for the node cut
  } else {
    n.rx = t.hx - r.a.x;
    n.ry = t.hy - r.a.y;
    n.rz = t.hz - r.a.z;
    const double q = n.rx * n.rx + n.ry * n.ry + n.rz * n.rz;
    n.n = q >= kCutR2 ? q * rsqrt(q) : 0.0;
  }
  return n;
}

template <class T>
struct SegV {
  T x, y, z;
};

template <class T, class Rec>
__device__ __forceinline__ void rec_fields(const Rec& r, T& gS, T& gH, SegV<T>& s0, SegV<T>& h0) {
  if constexpr (sizeof(T) == 4) {
    gS = r.hi.w;
    gH = r.lo.w;
    s0 = SegV<T>{r.sv.x, r.sv.y, r.sv.z};
    h0 = SegV<T>{r.sv.w, r.hv.x, r.hv.y};
  } else {
    gS = r.a.w;
    gH = r.b.x;
    s0 = SegV<T>{r.b.y, r.b.z, r.b.w};
    h0 = SegV<T>{r.c.x, r.c.y, r.c.z};
  }
}

// Segment start=A -> end=B at x (src/vortex.cpp:24-38): r1 = x - A,
// r2 = x - B, r0 = B - A, d = r1 x r2 = r0 x r1 and the reference's factor
// F = r0.(r1/|r1| - r2/|r2|) / |d|^2.  F is evaluated in forms that are
// algebraically equal to it but free of cancellation:
//   r1.r2 >= 0 (x beyond an end):  F = (|r1| + |r2|) / (|r1||r2| (|r1||r2| + r1.r2))
//   r1.r2 <  0 (x alongside):      F = (|r1| + |r2|) (|r1||r2| - r1.r2) / (|r1||r2| |d|^2)
// (the second from |r1|^2|r2|^2 - (r1.r2)^2 = |d|^2).  The reference form
// subtracts two nearly equal unit vectors when x is near the extension of the
// segment, which is where every wake node sees its lattice neighbours; in FP32
// that costs up to O(1) relative error there (1e-7 .. 1e-4 with these forms).
// Cut, as the reference does, when |d|^2 < 1e-10 or |x - A| < 1e-10 or
// |x - B| < 1e-10 (node_from marks such nodes with n = 0).  The node test is
// not implied by the |d|^2 test in FP32: for a stretched wake segment
// (|r0| ~ 10) whose end node is the target itself, the once-rounded r0 and
// x - A differ by an ulp and leave |d|^2 just above 1e-10.
template <class T>
__device__ __forceinline__ void seg(const SegV<T>& r0, const NodeV<T>& a, const NodeV<T>& b, T g, T& vx, T& vy,
                                    T& vz) {
  const T dx = r0.y * a.rz - r0.z * a.ry;
  const T dy = r0.z * a.rx - r0.x * a.rz;
  const T dz = r0.x * a.ry - r0.y * a.rx;
  const T d2 = dx * dx + dy * dy + dz * dz;
  const T dot12 = a.rx * b.rx + a.ry * b.ry + a.rz * b.rz;
  const T nn = a.n * b.n;
  const bool beyond = dot12 >= (T)0;
  const T num = (a.n + b.n) * (beyond ? (T)1 : nn - dot12);
  const T den = nn * (beyond ? nn + dot12 : d2);
  T k;
  if constexpr (sizeof(T) == 4) {
    k = g * num * nb_rcp(den);
  } else {
    k = g * num * __drcp_rn(den);
  }
  k = (d2 >= (T)kCutD2 && nn > (T)0) ? k : (T)0;
  vx += k * dx;
  vy += k * dy;
  vz += k * dz;
}

// Walk one staged strip for TPT targets: per node column, the H+1 node
// quantities, then the H chordwise segments of the column and the H spanwise
// segments that end in it.
template <class T, class Rec, int H, int TPT>
__device__ __forceinline__ void walk_strip(const Rec* sm, const StripInfo& si, const Tgt<T> (&tg)[TPT],
                                           T (&acc)[TPT][3]) {
  NodeV<T> prev[TPT][H];
  SegV<T> ps0[H];
  T pgS[H];
  const int nr = si.nr, n_rows = si.n_rows, n_cols = si.n_cols;
  for (int j = 0; j < n_cols; ++j) {
    NodeV<T> cur[TPT][H + 1];
    T gS[H], gH[H];
    SegV<T> s0[H], h0[H];
#pragma unroll
    for (int r = 0; r <= H; ++r) {
      if (r < nr) {
        const Rec rec = sm[r * n_cols + j];
        if (r < H) rec_fields<T, Rec>(rec, gS[r], gH[r], s0[r], h0[r]);
#pragma unroll
        for (int q = 0; q < TPT; ++q) cur[q][r] = node_from<T, Rec>(rec, tg[q]);
      }
    }
    const bool col_h = (j < n_cols - 1) || si.last_h;
#pragma unroll
    for (int r = 0; r < H; ++r) {
      if (r < n_rows && r + 1 < nr && col_h) {
#pragma unroll
        for (int q = 0; q < TPT; ++q) seg<T>(h0[r], cur[q][r], cur[q][r + 1], gH[r], acc[q][0], acc[q][1], acc[q][2]);
      }
    }
    if (j > 0) {
#pragma unroll
      for (int r = 0; r < H; ++r) {
        if (r < n_rows) {
#pragma unroll
          for (int q = 0; q < TPT; ++q) seg<T>(ps0[r], prev[q][r], cur[q][r], pgS[r], acc[q][0], acc[q][1], acc[q][2]);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < H; ++r) {
      if (r < n_rows) {
        pgS[r] = gS[r];
        ps0[r] = s0[r];
#pragma unroll
        for (int q = 0; q < TPT; ++q) prev[q][r] = cur[q][r];
      }
    }
  }
}

// One node column of a full strip (H owned node rows plus the row below,
// kStripCols + 1 columns, record stride kStripCols + 1 in shared memory): the
// node quantities of the column, its H chordwise segments (DO_H) and the H
// spanwise segments that end in it (!FIRST).  The column's quantities become
// `prev` for the next column; with the column loop unrolled by two the
// compiler renames instead of copying.
template <class T, class Rec, int H, int TPT, bool FIRST, bool DO_H>
__device__ __forceinline__ void full_column(const Rec* col, const Tgt<T> (&tg)[TPT], NodeV<T> (&prev)[TPT][H],
                                            SegV<T> (&ps0)[H], T (&pgS)[H], T (&acc)[TPT][3]) {
  NodeV<T> cur[TPT][H + 1];
  T gS[H], gH[H];
  SegV<T> s0[H], h0[H];
#pragma unroll
  for (int r = 0; r <= H; ++r) {
    const Rec rec = col[r * (kStripCols + 1)];
    if (r < H) rec_fields<T, Rec>(rec, gS[r], gH[r], s0[r], h0[r]);
#pragma unroll
    for (int q = 0; q < TPT; ++q) cur[q][r] = node_from<T, Rec>(rec, tg[q]);
  }
  if (DO_H) {
#pragma unroll
    for (int r = 0; r < H; ++r)
#pragma unroll
      for (int q = 0; q < TPT; ++q) seg<T>(h0[r], cur[q][r], cur[q][r + 1], gH[r], acc[q][0], acc[q][1], acc[q][2]);
  }
  if (!FIRST) {
#pragma unroll
    for (int r = 0; r < H; ++r)
#pragma unroll
      for (int q = 0; q < TPT; ++q) seg<T>(ps0[r], prev[q][r], cur[q][r], pgS[r], acc[q][0], acc[q][1], acc[q][2]);
  }
#pragma unroll
  for (int r = 0; r < H; ++r) {
    pgS[r] = gS[r];
    ps0[r] = s0[r];
#pragma unroll
    for (int q = 0; q < TPT; ++q) prev[q][r] = cur[q][r];
  }
}

// A full strip: compile-time bounds, no per-column predicates.  The last
// column owns its chordwise segments only at the sheet's last column.
template <class T, class Rec, int H, int TPT>
__device__ __forceinline__ void walk_full_strip(const Rec* sm, bool last_h, const Tgt<T> (&tg)[TPT],
                                                T (&acc)[TPT][3]) {
  NodeV<T> prev[TPT][H];
  SegV<T> ps0[H];
  T pgS[H];
  full_column<T, Rec, H, TPT, true, true>(sm, tg, prev, ps0, pgS, acc);
#pragma unroll 2
  for (int j = 1; j < kStripCols; ++j) full_column<T, Rec, H, TPT, false, true>(sm + j, tg, prev, ps0, pgS, acc);
  if (last_h)
    full_column<T, Rec, H, TPT, false, true>(sm + kStripCols, tg, prev, ps0, pgS, acc);
  else
    full_column<T, Rec, H, TPT, false, false>(sm + kStripCols, tg, prev, ps0, pgS, acc);
}

// ------------------------------------------------ packed FP32x2 walker
// The same arithmetic for the thread's two targets at once: lane .x is
// target 0, lane .y target 1, and every add/mul/fma is one sm_100 FP32x2
// instruction (__fadd2_rn / __fmul2_rn / __ffma2_rn) instead of two.  The
// reciprocal square roots, reciprocals and the per-lane selects stay scalar.
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

struct Node2 {
  float2 rx, ry, rz, n;
};

__device__ __forceinline__ float node_len(float q) { return q >= (float)kCutR2 ? q * nb_rsqrt(q) : 0.f; }

__device__ __forceinline__ Node2 node_from2(const RecF& r, const Tgt<float> (&tg)[2]) {
  const float2 thx = make_float2(tg[0].hx, tg[1].hx), thy = make_float2(tg[0].hy, tg[1].hy),
               thz = make_float2(tg[0].hz, tg[1].hz);
  const float2 tlx = make_float2(tg[0].lx, tg[1].lx), tly = make_float2(tg[0].ly, tg[1].ly),
               tlz = make_float2(tg[0].lz, tg[1].lz);
  Node2 n;
  n.rx = add2(add2(thx, bc2(-r.hi.x)), add2(tlx, bc2(-r.lo.x)));
  n.ry = add2(add2(thy, bc2(-r.hi.y)), add2(tly, bc2(-r.lo.y)));
  n.rz = add2(add2(thz, bc2(-r.hi.z)), add2(tlz, bc2(-r.lo.z)));
  const float2 q = fma2(n.rz, n.rz, fma2(n.ry, n.ry, mul2(n.rx, n.rx)));
  n.n = make_float2(node_len(q.x), node_len(q.y));
  return n;
}

// seg() for both lanes (same forms, same cut-offs).
__device__ __forceinline__ void seg2(const SegV<float>& r0, const Node2& a, const Node2& b, float g, float2& vx,
                                     float2& vy, float2& vz) {
  const float2 dx = fma2(bc2(r0.y), a.rz, mul2(bc2(-r0.z), a.ry));
  const float2 dy = fma2(bc2(r0.z), a.rx, mul2(bc2(-r0.x), a.rz));
  const float2 dz = fma2(bc2(r0.x), a.ry, mul2(bc2(-r0.y), a.rx));
  const float2 d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
  const float2 dot12 = fma2(a.rz, b.rz, fma2(a.ry, b.ry, mul2(a.rx, b.rx)));
  const float2 nn = mul2(a.n, b.n);
  const float2 sn = add2(a.n, b.n);
  const float2 tp = add2(nn, dot12);
  const float2 tm = fma2(dot12, bc2(-1.f), nn);
  const bool bx = dot12.x >= 0.f, by = dot12.y >= 0.f;
  const float2 num = mul2(sn, make_float2(bx ? 1.f : tm.x, by ? 1.f : tm.y));
  const float2 den = mul2(nn, make_float2(bx ? tp.x : d2.x, by ? tp.y : d2.y));
  float2 k = mul2(mul2(bc2(g), num), make_float2(nb_rcp(den.x), nb_rcp(den.y)));
  k.x = (d2.x >= (float)kCutD2 && nn.x > 0.f) ? k.x : 0.f;
  k.y = (d2.y >= (float)kCutD2 && nn.y > 0.f) ? k.y : 0.f;
  vx = fma2(k, dx, vx);
  vy = fma2(k, dy, vy);
  vz = fma2(k, dz, vz);
}

template <int H, bool FIRST, bool DO_H>
__device__ __forceinline__ void full_column2(const RecF* col, const Tgt<float> (&tg)[2], Node2 (&prev)[H],
                                             SegV<float> (&ps0)[H], float (&pgS)[H], float2 (&acc)[3]) {
  Node2 cur[H + 1];
  float gS[H], gH[H];
  SegV<float> s0[H], h0[H];
#pragma unroll
  for (int r = 0; r <= H; ++r) {
    const RecF rec = col[r * (kStripCols + 1)];
    if (r < H) rec_fields<float, RecF>(rec, gS[r], gH[r], s0[r], h0[r]);
    cur[r] = node_from2(rec, tg);
  }
  if (DO_H) {
#pragma unroll
    for (int r = 0; r < H; ++r) seg2(h0[r], cur[r], cur[r + 1], gH[r], acc[0], acc[1], acc[2]);
  }
  if (!FIRST) {
#pragma unroll
    for (int r = 0; r < H; ++r) seg2(ps0[r], prev[r], cur[r], pgS[r], acc[0], acc[1], acc[2]);
  }
#pragma unroll
  for (int r = 0; r < H; ++r) {
    pgS[r] = gS[r];
    ps0[r] = s0[r];
    prev[r] = cur[r];
  }
}

template <int H>
__device__ __forceinline__ void walk_full_strip2(const RecF* sm, bool last_h, const Tgt<float> (&tg)[2],
                                                 float (&acc)[2][3]) {
  Node2 prev[H];
  SegV<float> ps0[H];
  float pgS[H];
  float2 a2[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  full_column2<H, true, true>(sm, tg, prev, ps0, pgS, a2);
#pragma unroll 2
  for (int j = 1; j < kStripCols; ++j) full_column2<H, false, true>(sm + j, tg, prev, ps0, pgS, a2);
  if (last_h)
    full_column2<H, false, true>(sm + kStripCols, tg, prev, ps0, pgS, a2);
  else
    full_column2<H, false, false>(sm + kStripCols, tg, prev, ps0, pgS, a2);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    acc[0][c] += a2[c].x;
    acc[1][c] += a2[c].y;
  }
}

// ------------------------------------------- far-field packed walker
// A strip whose staged nodes all lie within rho of a local origin O (one of
// its own nodes) is "far" from a target x when |x - O| >= 2 rho + 1e-3.  Then
// every pair has |r| >= rho + 1e-3, so no node is cut (|r| > 1e-10) and every
// r1.r2 > 0 (the strip subtends less than 60 degrees from x), which leaves the
// beyond-end form of the segment factor alone, without cancellation; it is
// evaluated as 2 g (|r1|+|r2|) / (|r1||r2| ((|r1|+|r2|)^2 - |r0|^2)) with the
// segment's |r0|^2 from its record, which needs no r1.r2.  With
// node and target coordinates relative to O (FP32, rounded from the hi/lo
// differences), r = x_O - p_O costs one subtraction per component instead of
// three, and its error stays below ulp(rho)/2 + ulp(|x_O|)/2 <= 1.5 ulp(|r|).
// The cut |d|^2 < 1e-10 is kept (a far target can lie on a segment's line).
__device__ __forceinline__ Node2 node_far2(const float4 L, const float2 (&ts)[3]) {
  Node2 n;
  n.rx = add2(ts[0], bc2(-L.x));
  n.ry = add2(ts[1], bc2(-L.y));
  n.rz = add2(ts[2], bc2(-L.z));
  const float2 q = fma2(n.rz, n.rz, fma2(n.ry, n.ry, mul2(n.rx, n.rx)));
  n.n = mul2(q, make_float2(nb_rsqrt(q.x), nb_rsqrt(q.y)));
  return n;
}

__device__ __forceinline__ void seg_far2(const SegV<float>& r0, float l2, const Node2& a, const Node2& b, float g2,
                                         float2& vx, float2& vy, float2& vz) {
  const float2 dx = fma2(bc2(r0.y), a.rz, mul2(bc2(-r0.z), a.ry));
  const float2 dy = fma2(bc2(r0.z), a.rx, mul2(bc2(-r0.x), a.rz));
  const float2 dz = fma2(bc2(r0.x), a.ry, mul2(bc2(-r0.y), a.rx));
  const float2 d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
  // 2 (|r1||r2| + r1.r2) = (|r1| + |r2|)^2 - |r0|^2 (r1 - r2 = r0): no dot
  // product; in the far field |r1| + |r2| exceeds |r0| by a margin of the
  // strip's size, so the difference loses at most a couple of bits
  const float2 sn = add2(a.n, b.n);
  const float2 den = mul2(mul2(a.n, b.n), fma2(sn, sn, bc2(-l2)));
  float2 k = mul2(mul2(bc2(g2), sn), make_float2(nb_rcp(den.x), nb_rcp(den.y)));
  k.x = d2.x >= (float)kCutD2 ? k.x : 0.f;
  k.y = d2.y >= (float)kCutD2 ? k.y : 0.f;
  vx = fma2(k, dx, vx);
  vy = fma2(k, dy, vy);
  vz = fma2(k, dz, vz);
}

// One node column of a far strip: local node coordinates and 2 gS from
// `lcol`, the rest of the record (gH, segment vectors and their squared
// lengths) from `col`.  The spanwise segments ending in this column use the
// previous column's vectors, lengths and strengths (ps0, pl2, pgS).
template <int H, bool FIRST, bool DO_H>
__device__ __forceinline__ void far_column2(const RecF* col, const float4* lcol, const float2 (&ts)[3],
                                            Node2 (&prev)[H], SegV<float> (&ps0)[H], float (&pl2)[H],
                                            float (&pgS)[H], float2 (&acc)[3]) {
  Node2 cur[H + 1];
  float gS[H], gH[H], l2S[H], l2H[H];
  SegV<float> s0[H], h0[H];
#pragma unroll
  for (int r = 0; r <= H; ++r) {
    const float4 L = lcol[r * (kStripCols + 1)];
    if (r < H) {
      const RecF& rec = col[r * (kStripCols + 1)];
      const float4 sv = rec.sv, hv = rec.hv;
      const float gh = rec.lo.w;
      gS[r] = L.w;
      gH[r] = gh + gh;
      s0[r] = SegV<float>{sv.x, sv.y, sv.z};
      h0[r] = SegV<float>{sv.w, hv.x, hv.y};
      l2S[r] = hv.z;
      l2H[r] = hv.w;
    }
    cur[r] = node_far2(L, ts);
  }
  if (DO_H) {
#pragma unroll
    for (int r = 0; r < H; ++r) seg_far2(h0[r], l2H[r], cur[r], cur[r + 1], gH[r], acc[0], acc[1], acc[2]);
  }
  if (!FIRST) {
#pragma unroll
    for (int r = 0; r < H; ++r) seg_far2(ps0[r], pl2[r], prev[r], cur[r], pgS[r], acc[0], acc[1], acc[2]);
  }
#pragma unroll
  for (int r = 0; r < H; ++r) {
    pgS[r] = gS[r];
    ps0[r] = s0[r];
    pl2[r] = l2S[r];
    prev[r] = cur[r];
  }
}

// Column-bounded forms of the packed walkers: the strip's n_cols node
// columns (row-padded staging), the chordwise segments of the last column
// only when the strip owns them (last_h).
template <int H>
__device__ __forceinline__ void walk_cols2(const RecF* sm, int n_cols, bool last_h, const Tgt<float> (&tg)[2],
                                           float (&acc)[2][3]) {
  Node2 prev[H];
  SegV<float> ps0[H];
  float pgS[H];
  float2 a2[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  if (n_cols == 1) {
    if (last_h)
      full_column2<H, true, true>(sm, tg, prev, ps0, pgS, a2);
    else
      full_column2<H, true, false>(sm, tg, prev, ps0, pgS, a2);
  } else {
    full_column2<H, true, true>(sm, tg, prev, ps0, pgS, a2);
#pragma unroll 2
    for (int j = 1; j < n_cols - 1; ++j) full_column2<H, false, true>(sm + j, tg, prev, ps0, pgS, a2);
    if (last_h)
      full_column2<H, false, true>(sm + n_cols - 1, tg, prev, ps0, pgS, a2);
    else
      full_column2<H, false, false>(sm + n_cols - 1, tg, prev, ps0, pgS, a2);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    acc[0][c] += a2[c].x;
    acc[1][c] += a2[c].y;
  }
}

template <int H>
__device__ __forceinline__ void walk_far_cols2(const RecF* sm, const float4* loc, int n_cols, bool last_h,
                                               const float2 (&ts)[3], float (&acc)[2][3]) {
  Node2 prev[H];
  SegV<float> ps0[H];
  float pl2[H], pgS[H];
  float2 a2[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  if (n_cols == 1) {
    if (last_h)
      far_column2<H, true, true>(sm, loc, ts, prev, ps0, pl2, pgS, a2);
    else
      far_column2<H, true, false>(sm, loc, ts, prev, ps0, pl2, pgS, a2);
  } else {
    far_column2<H, true, true>(sm, loc, ts, prev, ps0, pl2, pgS, a2);
#pragma unroll 2
    for (int j = 1; j < n_cols - 1; ++j) far_column2<H, false, true>(sm + j, loc + j, ts, prev, ps0, pl2, pgS, a2);
    if (last_h)
      far_column2<H, false, true>(sm + n_cols - 1, loc + n_cols - 1, ts, prev, ps0, pl2, pgS, a2);
    else
      far_column2<H, false, false>(sm + n_cols - 1, loc + n_cols - 1, ts, prev, ps0, pl2, pgS, a2);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    acc[0][c] += a2[c].x;
    acc[1][c] += a2[c].y;
  }
}

// The far test is made for the two column halves of a strip, each against
// its own origin: a warp whose targets are far from one half only walks that
// half with the far-field walker and the other with the near one.  Halves
// share the middle node column c (the left half owns its spanwise segments
// up to c, the right half the chordwise segments of c onwards); a strip of
// fewer than 3 node columns is one part.
//
// Local coordinates of the part [j0, j1] of a staged strip relative to its
// central real node O: loc[k] = (p_k - O, 2 gS_k) for real nodes, (0, 0, 0,
// 2 gS_k) for the zero padding rows (whose segments have zero strength).
// Returns whether all of this warp's targets are far from the part
// (warp-uniform).  Every thread of the
// block calls it (it synchronises); `red` holds 2 floats per warp, `slot`
// picks this part's.
__device__ __forceinline__ const RecF& part_origin(const RecF* sm, const StripInfo& si, int j0, int j1) {
  return sm[((si.nr - 1) >> 1) * (kStripCols + 1) + j0 + ((j1 - j0) >> 1)];
}

// The targets relative to a part's origin O (FP32, rounded from the hi/lo differences).
__device__ __forceinline__ void part_targets(const RecF& o, const Tgt<float> (&tg)[2], float2 (&ts)[3]) {
  const float4 oh = o.hi, ol = o.lo;
  ts[0] = make_float2((tg[0].hx - oh.x) + (tg[0].lx - ol.x), (tg[1].hx - oh.x) + (tg[1].lx - ol.x));
  ts[1] = make_float2((tg[0].hy - oh.y) + (tg[0].ly - ol.y), (tg[1].hy - oh.y) + (tg[1].ly - ol.y));
  ts[2] = make_float2((tg[0].hz - oh.z) + (tg[0].lz - ol.z), (tg[1].hz - oh.z) + (tg[1].lz - ol.z));
}

template <int H, int BLOCK>
__device__ __forceinline__ bool far_prepare(const RecF* sm, const StripInfo& si, int j0, int j1, float4* loc,
                                            float* red, int slot, const Tgt<float> (&tg)[2]) {
  const int w = j1 - j0 + 1;
  const RecF& o = part_origin(sm, si, j0, j1);
  const float4 oh = o.hi, ol = o.lo;
  float m = 0.f;
  for (int q = threadIdx.x; q < (H + 1) * w; q += BLOCK) {
    const int r = q / w, j = j0 + (q - r * w);
    const int k = r * (kStripCols + 1) + j;
    const float4 h = sm[k].hi, l = sm[k].lo;
    float4 L = make_float4(0.f, 0.f, 0.f, h.w + h.w);  // 2 gS (the far segment factor's form)
    if (r < si.nr) {
      L.x = (h.x - oh.x) + (l.x - ol.x);
      L.y = (h.y - oh.y) + (l.y - ol.y);
      L.z = (h.z - oh.z) + (l.z - ol.z);
      m = fmaxf(m, fmaf(L.z, L.z, fmaf(L.y, L.y, L.x * L.x)));
    }
    loc[k] = L;
  }
#pragma unroll
  for (int off = 16; off; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) red[2 * (threadIdx.x >> 5) + slot] = m;
  __syncthreads();
  float rho2 = red[slot];
#pragma unroll
  for (int v = 1; v < BLOCK / 32; ++v) rho2 = fmaxf(rho2, red[2 * v + slot]);
  const float lim = 2.000001f * sqrtf(rho2) + 1e-3f;
  float2 ts[3];
  part_targets(o, tg, ts);
  const float2 t2 = fma2(ts[2], ts[2], fma2(ts[1], ts[1], mul2(ts[0], ts[0])));
  return __all_sync(0xffffffffu, t2.x >= lim * lim && t2.y >= lim * lim);
}

// ------------------------------------------------ far-field FP64 walker
// The far-field algebra for the FP64 form: a warp whose targets are at least
// 2 rho + 1e-3 from a part's central node O (rho: the part's radius about O)
// sees every node beyond rho + 1e-3 (none is cut) and every r1.r2 > 0, so the
// segment factor takes the single form 2 g (|r1|+|r2|) / (|r1||r2|
// ((|r1|+|r2|)^2 - |r0|^2)) (no r1.r2, no select); the |d|^2 < 1e-10 cut
// stays.  FP64 positions need no O-relative coordinates: r = x - p directly.
template <class T>
__device__ __forceinline__ void seg_far(const SegV<T>& r0, T l2, const NodeV<T>& a, const NodeV<T>& b, T g, T& vx,
                                        T& vy, T& vz) {
  const T dx = r0.y * a.rz - r0.z * a.ry;
  const T dy = r0.z * a.rx - r0.x * a.rz;
  const T dz = r0.x * a.ry - r0.y * a.rx;
  const T d2 = dx * dx + dy * dy + dz * dz;
  const T sn = a.n + b.n;
  const T den = a.n * b.n * (sn * sn - l2);
  T k = (g + g) * sn * __drcp_rn(den);
  k = d2 >= (T)kCutD2 ? k : (T)0;
  vx += k * dx;
  vy += k * dy;
  vz += k * dz;
}

template <class T, class Rec, int H, int TPT, bool FIRST, bool DO_H>
__device__ __forceinline__ void far_column(const Rec* col, const Tgt<T> (&tg)[TPT], NodeV<T> (&prev)[TPT][H],
                                           SegV<T> (&ps0)[H], T (&pl2)[H], T (&pgS)[H], T (&acc)[TPT][3]) {
  NodeV<T> cur[TPT][H + 1];
  T gS[H], gH[H], l2S[H], l2H[H];
  SegV<T> s0[H], h0[H];
#pragma unroll
  for (int r = 0; r <= H; ++r) {
    const Rec rec = col[r * (kStripCols + 1)];
    if (r < H) {
      rec_fields<T, Rec>(rec, gS[r], gH[r], s0[r], h0[r]);
      l2S[r] = s0[r].x * s0[r].x + s0[r].y * s0[r].y + s0[r].z * s0[r].z;
      l2H[r] = h0[r].x * h0[r].x + h0[r].y * h0[r].y + h0[r].z * h0[r].z;
    }
#pragma unroll
    for (int q = 0; q < TPT; ++q) cur[q][r] = node_from<T, Rec>(rec, tg[q]);
  }
  if (DO_H) {
#pragma unroll
    for (int r = 0; r < H; ++r)
#pragma unroll
      for (int q = 0; q < TPT; ++q)
        seg_far<T>(h0[r], l2H[r], cur[q][r], cur[q][r + 1], gH[r], acc[q][0], acc[q][1], acc[q][2]);
  }
  if (!FIRST) {
#pragma unroll
    for (int r = 0; r < H; ++r)
#pragma unroll
      for (int q = 0; q < TPT; ++q)
        seg_far<T>(ps0[r], pl2[r], prev[q][r], cur[q][r], pgS[r], acc[q][0], acc[q][1], acc[q][2]);
  }
#pragma unroll
  for (int r = 0; r < H; ++r) {
    pgS[r] = gS[r];
    ps0[r] = s0[r];
    pl2[r] = l2S[r];
#pragma unroll
    for (int q = 0; q < TPT; ++q) prev[q][r] = cur[q][r];
  }
}

// Column-bounded generic walkers over row-padded staging (record stride
// kStripCols + 1): the near-field one (full_column) or the far-field one.
template <class T, class Rec, int H, int TPT, bool FAR>
__device__ __forceinline__ void walk_cols(const Rec* sm, int n_cols, bool last_h, const Tgt<T> (&tg)[TPT],
                                          T (&acc)[TPT][3]) {
  NodeV<T> prev[TPT][H];
  SegV<T> ps0[H];
  T pl2[H], pgS[H];
  auto col = [&](const Rec* c, auto first, auto do_h) {
    constexpr bool kFirst = decltype(first)::value, kDoH = decltype(do_h)::value;
    if constexpr (FAR)
      far_column<T, Rec, H, TPT, kFirst, kDoH>(c, tg, prev, ps0, pl2, pgS, acc);
    else
      full_column<T, Rec, H, TPT, kFirst, kDoH>(c, tg, prev, ps0, pgS, acc);
  };
  using Yes = std::true_type;
  using No = std::false_type;
  if (n_cols == 1) {
    if (last_h)
      col(sm, Yes{}, Yes{});
    else
      col(sm, Yes{}, No{});
    return;
  }
  col(sm, Yes{}, Yes{});
#pragma unroll 2
  for (int j = 1; j < n_cols - 1; ++j) col(sm + j, No{}, Yes{});
  if (last_h)
    col(sm + n_cols - 1, No{}, Yes{});
  else
    col(sm + n_cols - 1, No{}, No{});
}

// Far test of the part [j0, j1] of a staged FP64 strip (every thread of the
// block calls it: it synchronises): the part's radius about its central node
// by a block max, then whether all of this warp's targets are far from it.
template <class Rec, int H, int BLOCK, int TPT>
__device__ __forceinline__ bool far_prepare_d(const Rec* sm, const StripInfo& si, int j0, int j1, float* red,
                                              int slot, const Tgt<double> (&tg)[TPT]) {
  const int w = j1 - j0 + 1;
  const Rec& o = sm[((si.nr - 1) >> 1) * (kStripCols + 1) + j0 + ((j1 - j0) >> 1)];
  const double ox = o.a.x, oy = o.a.y, oz = o.a.z;
  double m = 0.0;
  for (int q = threadIdx.x; q < si.nr * w; q += BLOCK) {
    const int r = q / w, j = j0 + (q - r * w);
    const Rec& p = sm[r * (kStripCols + 1) + j];
    const double dx = p.a.x - ox, dy = p.a.y - oy, dz = p.a.z - oz;
    m = fmax(m, dx * dx + dy * dy + dz * dz);
  }
  float mf = __double2float_ru(m);
#pragma unroll
  for (int off = 16; off; off >>= 1) mf = fmaxf(mf, __shfl_xor_sync(0xffffffffu, mf, off));
  if ((threadIdx.x & 31) == 0) red[2 * (threadIdx.x >> 5) + slot] = mf;
  __syncthreads();
  float rho2 = red[slot];
#pragma unroll
  for (int v = 1; v < BLOCK / 32; ++v) rho2 = fmaxf(rho2, red[2 * v + slot]);
  const double lim = 2.000001 * sqrt((double)rho2) + 1e-3;
  bool far = true;
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    const double dx = tg[q].hx - ox, dy = tg[q].hy - oy, dz = tg[q].hz - oz;
    far = far && (dx * dx + dy * dy + dz * dz >= lim * lim);
  }
  return __all_sync(0xffffffffu, far);
}

// ------------------------------------------------ FP64 near field
// The mixed form's near pairs (those the far-field test leaves to the
// near-field walker) in FP64 when the context asks for it: the plain FP64
// form's near-field arithmetic (seg<double>) on the FP64 records of the same
// sheets, read from global memory (they stay in L1/L2), for the thread's
// targets one at a time, accumulated in FP64.  Rows past the strip's loaded
// rows read as zero records, as the row-padded staging does.
template <int H, bool FIRST, bool DO_H>
__device__ __forceinline__ void near64_column(const RecD* __restrict__ col, int stride, int nr,
                                              const Tgt<double> (&tg)[1], NodeV<double> (&prev)[1][H],
                                              SegV<double> (&ps0)[H], double (&pgS)[H], double (&acc)[1][3]) {
  NodeV<double> cur[1][H + 1];
  double gS[H], gH[H];
  SegV<double> s0[H], h0[H];
#pragma unroll
  for (int r = 0; r <= H; ++r) {
    RecD rec;
    if (r < nr) {
      rec = col[(long long)r * stride];
    } else {
      rec.a = make_double4(0, 0, 0, 0);
      rec.b = rec.a;
      rec.c = rec.a;
    }
    if (r < H) rec_fields<double, RecD>(rec, gS[r], gH[r], s0[r], h0[r]);
    cur[0][r] = node_from<double, RecD>(rec, tg[0]);
  }
  if (DO_H) {
#pragma unroll
    for (int r = 0; r < H; ++r) seg<double>(h0[r], cur[0][r], cur[0][r + 1], gH[r], acc[0][0], acc[0][1], acc[0][2]);
  }
  if (!FIRST) {
#pragma unroll
    for (int r = 0; r < H; ++r) seg<double>(ps0[r], prev[0][r], cur[0][r], pgS[r], acc[0][0], acc[0][1], acc[0][2]);
  }
#pragma unroll
  for (int r = 0; r < H; ++r) {
    pgS[r] = gS[r];
    ps0[r] = s0[r];
    prev[0][r] = cur[0][r];
  }
}

// Columns [0, n_cols) of a part starting at `base` (record of its first
// row); the chordwise segments of the last column only when owned.
template <int H>
__device__ __forceinline__ void walk_near64(const RecD* __restrict__ base, int stride, int nr, int n_cols, bool last_h,
                                            const Tgt<double> (&tg)[1], double (&acc)[1][3]) {
  NodeV<double> prev[1][H];
  SegV<double> ps0[H];
  double pgS[H];
  if (n_cols == 1) {
    if (last_h)
      near64_column<H, true, true>(base, stride, nr, tg, prev, ps0, pgS, acc);
    else
      near64_column<H, true, false>(base, stride, nr, tg, prev, ps0, pgS, acc);
    return;
  }
  near64_column<H, true, true>(base, stride, nr, tg, prev, ps0, pgS, acc);
#pragma unroll 1
  for (int j = 1; j < n_cols - 1; ++j) near64_column<H, false, true>(base + j, stride, nr, tg, prev, ps0, pgS, acc);
  if (last_h)
    near64_column<H, false, true>(base + n_cols - 1, stride, nr, tg, prev, ps0, pgS, acc);
  else
    near64_column<H, false, false>(base + n_cols - 1, stride, nr, tg, prev, ps0, pgS, acc);
}

// Targets tile0 + threadIdx.x + q BLOCK (clamped to the last one) of the
// SoA arrays, as hi/lo FP32 pairs or FP64.
template <class T, int TPT, int BLOCK>
__device__ __forceinline__ void load_targets(const double* __restrict__ tx, const double* __restrict__ ty,
                                             const double* __restrict__ tz, long long base, long long tile0,
                                             long long n_targets, Tgt<T> (&tg)[TPT]) {
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    long long t = tile0 + threadIdx.x + (long long)q * BLOCK;
    if (t >= n_targets) t = n_targets - 1;  // padded lanes recompute the last target
    const double x = tx[base + t], y = ty[base + t], z = tz[base + t];
    if constexpr (sizeof(T) == 4) {
      tg[q].hx = (float)x; tg[q].hy = (float)y; tg[q].hz = (float)z;
      tg[q].lx = (float)(x - (double)tg[q].hx);
      tg[q].ly = (float)(y - (double)tg[q].hy);
      tg[q].lz = (float)(z - (double)tg[q].hz);
    } else {
      tg[q].hx = x; tg[q].hy = y; tg[q].hz = z;
      tg[q].lx = tg[q].ly = tg[q].lz = 0;
    }
  }
}

// Strips [s_begin, s_end) of B for the thread's targets, double-buffered
// through shared memory; FP32 partial sums per strip, FP64 across strips.
// PK: 0 generic walkers, 1 packed FP32x2 walker on full strips, 2 the packed
// walkers bounded by each strip's column count (row-padded staging, any
// fill) with the far-field walker for strips far from all of a warp's
// targets (`loc`, `red`: its shared-memory scratch).
template <class T, class Rec, int H, int TPT, int BLOCK, bool PAD, int PK = 0, bool NEAR64 = false>
__device__ __forceinline__ void eval_strips(const Blocks& B, long long s_begin, long long s_end,
                                            const Rec* __restrict__ rec, Rec* buf0, Rec* buf1, float4* loc,
                                            float* red, const Tgt<T> (&tg)[TPT], double (&accd)[TPT][3],
                                            const RecD* __restrict__ rec64 = nullptr, long long s_stride = 1) {
  if (s_begin >= s_end) return;
  StripInfo si = decode_strip<H>(B, s_begin);
  if constexpr (PAD && PK == 2)
    stage_strip_rows<Rec, H>(buf0, rec, si);
  else if constexpr (PAD)
    stage_strip_padded<Rec, H>(buf0, rec, si);
  else
    stage_strip<Rec>(buf0, rec, si);
  long long it = 0;
  for (long long s = s_begin; s < s_end; s += s_stride, ++it) {
    Rec* cur = (it & 1) ? buf1 : buf0;
    Rec* nxt = (it & 1) ? buf0 : buf1;
    StripInfo sn;
    const bool has_next = s + s_stride < s_end;
    if (has_next) {
      sn = decode_strip<H>(B, s + s_stride);
      if constexpr (PAD && PK == 2)
        stage_strip_rows<Rec, H>(nxt, rec, sn);
      else if constexpr (PAD)
        stage_strip_padded<Rec, H>(nxt, rec, sn);
      else
        stage_strip<Rec>(nxt, rec, sn);
      asm volatile("cp.async.wait_group 1;");
    } else {
      asm volatile("cp.async.wait_group 0;");
    }
    __syncthreads();
    T acc[TPT][3];
#pragma unroll
    for (int q = 0; q < TPT; ++q) acc[q][0] = acc[q][1] = acc[q][2] = (T)0;
    if constexpr (PAD && PK == 2 && sizeof(T) == 4 && TPT == 2) {
      const int n = si.n_cols;
      const int c = n >= 3 ? n >> 1 : n - 1;  // the parts [0, c] and [c, n - 1] (the second empty if c = n - 1)
      float4* locr = loc + (H + 1) * (kStripCols + 1);
      const bool farl = far_prepare<H, BLOCK>(cur, si, 0, c, loc, red, 0, tg);
      const bool farr = c < n - 1 && far_prepare<H, BLOCK>(cur, si, c, n - 1, locr, red, 1, tg);
      // one part when the strip is not split or both halves are near, else the two halves
      const bool one = c == n - 1 || (!farl && !farr);
#pragma unroll 1
      for (int p = 0; p < (one ? 1 : 2); ++p) {
        const int j0 = p ? c : 0, nc = one ? n : (p ? n - c : c + 1);
        const bool lh = (one || p) ? si.last_h : false;
        if (p ? farr : farl) {
          float2 ts[3];
          part_targets(part_origin(cur, si, j0, j0 + nc - 1), tg, ts);
          walk_far_cols2<H>(cur + j0, (p ? locr : loc) + j0, nc, lh, ts, acc);
        } else if constexpr (NEAR64) {
          // near part in FP64 from the FP64 records, one target at a time
#pragma unroll 1
          for (int q = 0; q < 2; ++q) {
            Tgt<double> td[1];
            td[0].hx = (double)tg[q].hx + (double)tg[q].lx;
            td[0].hy = (double)tg[q].hy + (double)tg[q].ly;
            td[0].hz = (double)tg[q].hz + (double)tg[q].lz;
            td[0].lx = td[0].ly = td[0].lz = 0.0;
            double a64[1][3] = {{0.0, 0.0, 0.0}};
            walk_near64<H>(rec64 + si.first + j0, si.row_stride, si.nr, nc, lh, td, a64);
            accd[q][0] += a64[0][0];
            accd[q][1] += a64[0][1];
            accd[q][2] += a64[0][2];
          }
        } else {
          walk_cols2<H>(cur + j0, nc, lh, tg, acc);
        }
      }
    } else if constexpr (PAD && PK == 2 && sizeof(T) == 8) {
      // FP64 form: the two column halves of the strip, each walked by the
      // far-field walker when every target of the warp is far from it
      const int n = si.n_cols;
      const int c = n >= 3 ? n >> 1 : n - 1;
      const bool farl = far_prepare_d<Rec, H, BLOCK, TPT>(cur, si, 0, c, red, 0, tg);
      const bool farr = c < n - 1 && far_prepare_d<Rec, H, BLOCK, TPT>(cur, si, c, n - 1, red, 1, tg);
      const bool one = c == n - 1 || (!farl && !farr);
#pragma unroll 1
      for (int p = 0; p < (one ? 1 : 2); ++p) {
        const int j0 = p ? c : 0, nc = one ? n : (p ? n - c : c + 1);
        const bool lh = (one || p) ? si.last_h : false;
        if (p ? farr : farl)
          walk_cols<T, Rec, H, TPT, true>(cur + j0, nc, lh, tg, acc);
        else
          walk_cols<T, Rec, H, TPT, false>(cur + j0, nc, lh, tg, acc);
      }
    } else if constexpr (PAD && PK == 1 && sizeof(T) == 4 && TPT == 2) {
      walk_full_strip2<H>(cur, si.last_h, tg, acc);
    } else if constexpr (PAD)
      walk_full_strip<T, Rec, H, TPT>(cur, si.last_h, tg, acc);
    else
      walk_strip<T, Rec, H, TPT>(cur, si, tg, acc);
#pragma unroll
    for (int q = 0; q < TPT; ++q) {
      accd[q][0] += (double)acc[q][0];
      accd[q][1] += (double)acc[q][1];
      accd[q][2] += (double)acc[q][2];
    }
    __syncthreads();  // everyone done with `cur` before it is refilled
    if (has_next) si = sn;
  }
}

template <class T, class Rec, int H, int TPT, int BLOCK, int MINB, bool PAD, int PK, bool NEAR64 = false>
__global__ void __launch_bounds__(BLOCK, MINB) nbody_kernel(Blocks B, long long n_strips,
                                                       const double* __restrict__ tx, const double* __restrict__ ty,
                                                       const double* __restrict__ tz, long long n_targets,
                                                       const Rec* __restrict__ rec, double* __restrict__ partial,
                                                       const RecD* __restrict__ rec64) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Rec* buf0 = reinterpret_cast<Rec*>(smem_raw);
  Rec* buf1 = buf0 + (H + 1) * (kStripCols + 1);
  float4* loc = reinterpret_cast<float4*>(buf1 + (H + 1) * (kStripCols + 1));
  // the FP32 far-field walker's local coordinates (none in the FP64 form), then the per-warp maxima
  float* red = reinterpret_cast<float*>(loc + (sizeof(Rec) == sizeof(RecF) ? 2 * (H + 1) * (kStripCols + 1) : 0));

  const long long tile0 = (long long)blockIdx.x * BLOCK * TPT;
  Tgt<T> tg[TPT];
  double accd[TPT][3];
  load_targets<T, TPT, BLOCK>(tx, ty, tz, 0, tile0, n_targets, tg);
#pragma unroll
  for (int q = 0; q < TPT; ++q) accd[q][0] = accd[q][1] = accd[q][2] = 0.0;
  // split y takes the strips y, y + splits, y + 2 splits, ...: the strips
  // near a target tile (the newest wake rows, next to the wing) are spread
  // over the splits instead of all landing in split 0, which evens out the
  // costlier near-field work
  eval_strips<T, Rec, H, TPT, BLOCK, PAD, PK, NEAR64>(B, (long long)blockIdx.y, n_strips, rec, buf0, buf1, loc, red,
                                                      tg, accd, rec64, (long long)gridDim.y);
  double* px = partial + (long long)blockIdx.y * 3 * n_targets;
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    const long long t = tile0 + threadIdx.x + (long long)q * BLOCK;
    if (t < n_targets) {
      px[t] = accd[q][0];
      px[n_targets + t] = accd[q][1];
      px[2 * n_targets + t] = accd[q][2];
    }
  }
}

// ------------------------------------------------------ batched evaluation
// Plans of all problems: strips, tiles, splits and the exclusive prefixes of
// items, partial sums and targets.  One CTA; a blockwide scan in chunks.
// select: -1 all problems, 0 only the general class, 1 only the padded class
// (the others get no targets, hence no items and no reduction).
template <int H, int TPC>
__global__ void __launch_bounds__(256) batch_plan_kernel(const NBodyBatchInput* __restrict__ in, int n, int select,
                                                         NBodyBatchPlan* __restrict__ plan, long long partial_cap,
                                                         long long* totals, int* status) {
  __shared__ long long sh[3][256];
  __shared__ long long carry[3];
  if (threadIdx.x < 3) carry[threadIdx.x] = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 256) {
    const int c = base + threadIdx.x;
    long long v[3] = {0, 0, 0};
    NBodyBatchPlan p{};
    if (c < n) {
      const NBodyBatchInput& x = in[c];
      const bool take = select < 0 || (int)batch_input_padded(x) == select;
      p.n_strips = fill_blocks(p.B, x.blocks, x.n_blocks, H);
      p.tgt_off = x.tgt_off;
      p.n_tgt = take ? x.n_tgt : 0;
      p.tiles = (p.n_tgt + TPC - 1) / TPC;
      p.splits = (p.n_strips + kBatchStripsPerItem - 1) / kBatchStripsPerItem;
      v[0] = p.tiles * p.splits;
      v[1] = p.splits * 3 * p.n_tgt;
      v[2] = p.n_tgt;
    }
    for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    // Hillis-Steele inclusive scan of the three counters
    for (int off = 1; off < 256; off <<= 1) {
      long long t[3];
      for (int k = 0; k < 3; ++k) t[k] = threadIdx.x >= off ? sh[k][threadIdx.x - off] : 0;
      __syncthreads();
      for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += t[k];
      __syncthreads();
    }
    if (c < n) {
      p.item_off = carry[0] + sh[0][threadIdx.x] - v[0];
      p.part_off = carry[1] + sh[1][threadIdx.x] - v[1];
      p.tgt_prefix = carry[2] + sh[2][threadIdx.x] - v[2];
      plan[c] = p;
    }
    __syncthreads();
    if (threadIdx.x < 3) carry[threadIdx.x] += sh[threadIdx.x][255];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const bool fits = carry[1] <= partial_cap;
    // an over-full plan evaluates and reduces nothing (the status reports it)
    totals[0] = fits ? carry[0] : 0;
    totals[1] = carry[1];
    totals[2] = fits ? carry[2] : 0;
    if (!fits) status[0] = 1;
  }
}

// Last problem whose prefix (member at `Off`) is <= w.
template <class F>
__device__ inline int plan_search(const NBodyBatchPlan* plan, int n, long long w, F key) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (key(plan[mid]) <= w)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

template <class T, class Rec, int H, int TPT, int BLOCK, int MINB, bool PAD, int PK>
__global__ void __launch_bounds__(BLOCK, MINB) batch_nbody_kernel(const NBodyBatchPlan* __restrict__ plan, int n,
                                                             const long long* __restrict__ totals,
                                                             const double* __restrict__ tx,
                                                             const double* __restrict__ ty,
                                                             const double* __restrict__ tz,
                                                             const Rec* __restrict__ rec,
                                                             double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Rec* buf0 = reinterpret_cast<Rec*>(smem_raw);
  Rec* buf1 = buf0 + (H + 1) * (kStripCols + 1);
  float4* loc = reinterpret_cast<float4*>(buf1 + (H + 1) * (kStripCols + 1));
  // the FP32 far-field walker's local coordinates (none in the FP64 form), then the per-warp maxima
  float* red = reinterpret_cast<float*>(loc + (sizeof(Rec) == sizeof(RecF) ? 2 * (H + 1) * (kStripCols + 1) : 0));
  const long long items = totals[0];
  for (long long w = blockIdx.x; w < items; w += gridDim.x) {
    const int c = plan_search(plan, n, w, [](const NBodyBatchPlan& p) { return p.item_off; });
    const NBodyBatchPlan& P = plan[c];
    const long long local = w - P.item_off;
    const long long tile = local / P.splits, split = local % P.splits;
    const long long tile0 = tile * BLOCK * TPT;
    Tgt<T> tg[TPT];
    double accd[TPT][3];
    load_targets<T, TPT, BLOCK>(tx, ty, tz, P.tgt_off, tile0, P.n_tgt, tg);
#pragma unroll
    for (int q = 0; q < TPT; ++q) accd[q][0] = accd[q][1] = accd[q][2] = 0.0;
    // interleaved source strips (split s: strips s, s + splits, ...), as in
    // nbody_kernel: a tile's near strips spread over its items
    eval_strips<T, Rec, H, TPT, BLOCK, PAD, PK>(P.B, split, P.n_strips, rec, buf0, buf1, loc, red, tg, accd, nullptr,
                                                P.splits);
    double* px = partial + P.part_off + split * 3 * P.n_tgt;
#pragma unroll
    for (int q = 0; q < TPT; ++q) {
      const long long t = tile0 + threadIdx.x + (long long)q * BLOCK;
      if (t < P.n_tgt) {
        px[t] = accd[q][0];
        px[P.n_tgt + t] = accd[q][1];
        px[2 * P.n_tgt + t] = accd[q][2];
      }
    }
  }
}

__global__ void batch_reduce_kernel(const NBodyBatchPlan* __restrict__ plan, int n,
                                    const long long* __restrict__ totals, const double* __restrict__ partial,
                                    double* vx, double* vy, double* vz) {
  const long long total = totals[2];
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    const int c = plan_search(plan, n, g, [](const NBodyBatchPlan& p) { return p.tgt_prefix; });
    const NBodyBatchPlan& P = plan[c];
    const long long t = g - P.tgt_prefix;
    double x = 0, y = 0, z = 0;
    for (long long s = 0; s < P.splits; ++s) {
      const double* p = partial + P.part_off + s * 3 * P.n_tgt;
      x += p[t];
      y += p[P.n_tgt + t];
      z += p[2 * P.n_tgt + t];
    }
    vx[P.tgt_off + t] = x;
    vy[P.tgt_off + t] = y;
    vz[P.tgt_off + t] = z;
  }
}

// Batched tiles: FP32 column-bounded packed FP32x2 h3 t2 b128 (every
// problem), FP64 h2 t1 b128; 3 CTAs/SM each.
constexpr int kBatchBlock = 128;
constexpr int kBatchTptF = 2, kBatchHFP = 3, kBatchTptD = 1, kBatchHD = 2, kBatchMinB = 3;
constexpr int kBatchPadPK = 2;  // walker of the padded class (see eval_strips)

__global__ void reduce_partials_kernel(const double* __restrict__ partial, int splits, long long n, double* vx,
                                       double* vy, double* vz) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    double x = 0, y = 0, z = 0;
    for (int s = 0; s < splits; ++s) {
      const double* p = partial + (long long)s * 3 * n;
      x += p[t];
      y += p[n + t];
      z += p[2 * n + t];
    }
    vx[t] = x;
    vy[t] = y;
    vz[t] = z;
  }
}

// ------------------------------------------------------------- variants
struct Variant {
  const char* name;
  int prec;  // NBodyPrec
  int H, TPT, BLOCK, MINB;
  int packed;  // 1: FP32x2 walker for full strips (FP32, TPT = 2); 2: plus the far-field walker
};

// Tile shapes: H owned node rows per strip, TPT targets per thread, BLOCK
// threads, MINB resident CTAs per SM requested from the register allocator.
constexpr Variant kVariants[] = {
    {"fp64_h4_t1_b128", kNBodyFP64, 4, 1, 128, 1, 0},
    {"fp64_h2_t1_b256", kNBodyFP64, 2, 1, 256, 1, 0},
    {"fp32_h4_t1_b256", kNBodyFP32, 4, 1, 256, 2, 0},
    {"fp32_h4_t2_b128", kNBodyFP32, 4, 2, 128, 3, 0},
    {"fp32_h2_t2_b128", kNBodyFP32, 2, 2, 128, 3, 0},
    {"fp32_h4_t1_b128_m4", kNBodyFP32, 4, 1, 128, 4, 0},
    {"fp32_h3_t2_b128_m4", kNBodyFP32, 3, 2, 128, 4, 0},
    {"fp32_h2_t1_b256_m3", kNBodyFP32, 2, 1, 256, 3, 0},
    {"fp64_h2_t2_b128", kNBodyFP64, 2, 2, 128, 1, 0},
    {"fp64_h2_t1_b128_m3", kNBodyFP64, 2, 1, 128, 3, 0},
    {"fp64_h2_t1_b256_m2", kNBodyFP64, 2, 1, 256, 2, 0},
    {"fp32_h3_t2_b128", kNBodyFP32, 3, 2, 128, 3, 0},
    {"fp32_h4_t2_b128_x2", kNBodyFP32, 4, 2, 128, 3, 1},
    {"fp32_h3_t2_b128_x2", kNBodyFP32, 3, 2, 128, 3, 1},
    {"fp32_h2_t2_b128_x2", kNBodyFP32, 2, 2, 128, 3, 1},
    {"fp32_h4_t2_b128_x2f", kNBodyFP32, 4, 2, 128, 3, 2},
    {"fp32_h3_t2_b128_x2f", kNBodyFP32, 3, 2, 128, 3, 2},
    {"fp32_h2_t2_b128_x2f", kNBodyFP32, 2, 2, 128, 3, 2},
    {"fp64_h2_t1_b128_m3f", kNBodyFP64, 2, 1, 128, 3, 2},
    {"fp64_h3_t1_b128_m2f", kNBodyFP64, 3, 1, 128, 2, 2},
    {"fp64_h2_t2_b128_f", kNBodyFP64, 2, 2, 128, 1, 2},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

// Full-tile (padded) walking pays when the sheets fill most of the padded
// columns: a sheet of C rings per row uses C + chunks of the chunks x
// (kStripCols + 1) staged node columns.
bool use_padded(const Blocks& B) {
  for (int i = 0; i < B.n; ++i) {
    const long long real = B.b[i].cols + B.chunks[i];
    const long long staged = (long long)B.chunks[i] * (kStripCols + 1);
    if (4 * real < 3 * staged) return false;
  }
  return true;
}

// Dynamic shared memory of a tile: two strip buffers, plus the far-field
// walker's local coordinates of the two halves and two per-warp maxima
// (PK == 2).
template <class Rec, int H, int BLOCK, int PK>
constexpr size_t strip_smem() {
  constexpr bool fp32 = sizeof(Rec) == sizeof(RecF);
  return 2 * sizeof(Rec) * (H + 1) * (kStripCols + 1) +
         (PK == 2 ? (fp32 ? 2 * sizeof(float4) * (H + 1) * (kStripCols + 1) : 0) + 2 * sizeof(float) * (BLOCK / 32)
                  : 0);
}

template <class T, class Rec, int H, int TPT, int BLOCK, int MINB, int PK = 0>
Error launch_variant(const Blocks& B, long long n_strips, const double* tx, const double* ty, const double* tz,
                     long long n_targets, const Rec* rec, NBodyWork* work, double* vx, double* vy, double* vz,
                     int num_sms, cudaStream_t st) {
  // the column-bounded walkers (PK == 2) take every sheet; the others pad only
  // sheets that fill most of the staged columns
  const bool pad = PK == 2 || use_padded(B);
  // the mixed form's near pairs in FP64 (packed FP32x2 tiles with the far-field walker)
  constexpr bool kCanNear64 = PK == 2 && sizeof(T) == 4 && TPT == 2;
  const RecD* rec64 = (kCanNear64 && work->near64) ? reinterpret_cast<const RecD*>(work->records64) : nullptr;
  if (kCanNear64 && work->near64 && !rec64) return fail(kErrInvalid, "FP64 near field without FP64 records");
  void (*kern)(Blocks, long long, const double*, const double*, const double*, long long, const Rec*, double*,
               const RecD*);
  if constexpr (kCanNear64)
    kern = rec64 ? nbody_kernel<T, Rec, H, TPT, BLOCK, MINB, true, PK, true>
                 : nbody_kernel<T, Rec, H, TPT, BLOCK, MINB, true, PK, false>;
  else if constexpr (PK == 2)
    kern = nbody_kernel<T, Rec, H, TPT, BLOCK, MINB, true, PK>;
  else
    kern = pad ? nbody_kernel<T, Rec, H, TPT, BLOCK, MINB, true, PK> : nbody_kernel<T, Rec, H, TPT, BLOCK, MINB, false, PK>;
  const size_t smem = strip_smem<Rec, H, BLOCK, PK>();
  // the shared-memory limit is a per-device attribute: set it once on every
  // device this process launches on (per kernel instance)
  static PerDeviceOnce attr_once[4];
  const int inst = (pad ? 1 : 0) + (rec64 ? 2 : 0);
  int dev = 0;
  UVLM_CUDA_TRY(cudaGetDevice(&dev));
  cudaError_t attr_err = cudaSuccess;
  if (!once_on_device(attr_once[inst], dev, [&] {
        attr_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        return attr_err == cudaSuccess;
      }))
    return fail(kErrCuda, std::string("nbody: the shared-memory attribute could not be set on this device") +
                              (attr_err != cudaSuccess ? std::string(": ") + cudaGetErrorString(attr_err) : ""));
  int occ = 0;
  UVLM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, BLOCK, smem));
  if (occ < 1) occ = 1;
  const long long tiles = (n_targets + (long long)BLOCK * TPT - 1) / ((long long)BLOCK * TPT);
  // enough CTAs for ~4 waves, but never more splits than strips
  const long long want = (long long)num_sms * occ * 4;
  long long splits = (want + tiles - 1) / tiles;
  if (splits > n_strips) splits = n_strips;
  if (splits > 64) splits = 64;
  if (work->max_splits > 0 && splits > work->max_splits) splits = work->max_splits;
  // never more splits than the partial-sum buffer holds for these targets
  if (splits > work->partial_cap / (3 * n_targets)) splits = work->partial_cap / (3 * n_targets);
  if (splits < 1) splits = 1;
  const long long sps = (n_strips + splits - 1) / splits;
  splits = (n_strips + sps - 1) / sps;
  const long long need = splits * 3 * n_targets;
  if (work->partial_cap < need) return fail(kErrCapacity, "nbody partial buffer too small");
  dim3 grid((unsigned)tiles, (unsigned)splits);
  kern<<<grid, BLOCK, smem, st>>>(B, n_strips, tx, ty, tz, n_targets, rec, work->partial, rec64);
  UVLM_LAUNCH_CHECK();
  const int rb = 256;
  const int rg = (int)std::min<long long>((n_targets + rb - 1) / rb, (long long)num_sms * 8);
  reduce_partials_kernel<<<rg, rb, 0, st>>>(work->partial, (int)splits, n_targets, vx, vy, vz);
  UVLM_LAUNCH_CHECK();
  return ok();
}

}  // namespace

int nbody_num_variants() { return kNumVariants; }
int nbody_variant_prec(int v) { return (v >= 0 && v < kNumVariants) ? kVariants[v].prec : -1; }
bool nbody_variant_near64(int v) {
  return v >= 0 && v < kNumVariants && kVariants[v].prec == kNBodyFP32 && kVariants[v].packed == 2 &&
         kVariants[v].TPT == 2;
}
const char* nbody_variant_name(int v) { return (v >= 0 && v < kNumVariants) ? kVariants[v].name : "?"; }

long long nbody_unique_segments(const SourceBlock* blocks, int n_blocks) {
  long long s = 0;
  for (int i = 0; i < n_blocks; ++i) {
    const long long R = blocks[i].node_rows - 1, C = blocks[i].cols;
    if (R < 0) continue;
    s += (long long)blocks[i].num * ((R + 1) * C + R * (C + 1));
  }
  return s;
}

Error nbody_build_sources(const SheetView* views, int n_views, NBodyPrec prec, NBodyWork* work,
                          SourceBlock* blocks, cudaStream_t st) {
  long long off = 0;
  const size_t rsz = prec == kNBodyFP32 ? sizeof(RecF) : sizeof(RecD);
  for (int i = 0; i < n_views; ++i) {
    const SheetView& v = views[i];
    const long long cnt = (long long)v.num * v.node_rows * (v.cols + 1);
    blocks[i] = SourceBlock{off, v.num, v.node_rows, v.cols};
    if ((off + cnt) * (long long)rsz > work->records_cap) return fail(kErrCapacity, "nbody record buffer too small");
    if (cnt > 0) {
      const int bs = 256;
      const int gs = (int)std::min<long long>((cnt + bs - 1) / bs, 4096);
      if (prec == kNBodyFP32)
        build_records_kernel<RecF><<<gs, bs, 0, st>>>(v, reinterpret_cast<RecF*>(work->records) + off);
      else
        build_records_kernel<RecD><<<gs, bs, 0, st>>>(v, reinterpret_cast<RecD*>(work->records) + off);
      UVLM_LAUNCH_CHECK();
      if (prec == kNBodyFP32 && work->near64) {
        // FP64 records of the same nodes for the FP64 near field
        if ((off + cnt) * (long long)sizeof(RecD) > work->records64_cap)
          return fail(kErrCapacity, "nbody FP64 record buffer too small");
        build_records_kernel<RecD><<<gs, bs, 0, st>>>(v, reinterpret_cast<RecD*>(work->records64) + off);
        UVLM_LAUNCH_CHECK();
      }
    }
    off += cnt;
  }
  return ok();
}

Error nbody_eval(const SourceBlock* blocks, int n_blocks, NBodyPrec prec, const double* tx, const double* ty,
                 const double* tz, long long n_targets, double* vx, double* vy, double* vz, NBodyWork* work,
                 int variant, int num_sms, cudaStream_t st) {
  if (n_targets <= 0) return ok();
  if (variant < 0 || variant >= kNumVariants || kVariants[variant].prec != prec)
    return fail(kErrInvalid, "nbody variant does not match precision");
  const Variant& V = kVariants[variant];
  Blocks B{};
  const long long strips = fill_blocks(B, blocks, n_blocks, V.H);
  if (strips == 0) {
    UVLM_CUDA_TRY(cudaMemsetAsync(vx, 0, sizeof(double) * n_targets, st));
    UVLM_CUDA_TRY(cudaMemsetAsync(vy, 0, sizeof(double) * n_targets, st));
    UVLM_CUDA_TRY(cudaMemsetAsync(vz, 0, sizeof(double) * n_targets, st));
    return ok();
  }
  const RecF* rf = reinterpret_cast<const RecF*>(work->records);
  const RecD* rd = reinterpret_cast<const RecD*>(work->records);
  const Blocks& B_ = B;
  switch (variant) {
    case 0: return launch_variant<double, RecD, 4, 1, 128, 1>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 1: return launch_variant<double, RecD, 2, 1, 256, 1>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 2: return launch_variant<float, RecF, 4, 1, 256, 2>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 3: return launch_variant<float, RecF, 4, 2, 128, 3>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 4: return launch_variant<float, RecF, 2, 2, 128, 3>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 5: return launch_variant<float, RecF, 4, 1, 128, 4>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 6: return launch_variant<float, RecF, 3, 2, 128, 4>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 7: return launch_variant<float, RecF, 2, 1, 256, 3>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 8: return launch_variant<double, RecD, 2, 2, 128, 1>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 9: return launch_variant<double, RecD, 2, 1, 128, 3>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 10: return launch_variant<double, RecD, 2, 1, 256, 2>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 11: return launch_variant<float, RecF, 3, 2, 128, 3>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 12: return launch_variant<float, RecF, 4, 2, 128, 3, 1>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 13: return launch_variant<float, RecF, 3, 2, 128, 3, 1>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 14: return launch_variant<float, RecF, 2, 2, 128, 3, 1>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 15: return launch_variant<float, RecF, 4, 2, 128, 3, 2>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 16: return launch_variant<float, RecF, 3, 2, 128, 3, 2>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 17: return launch_variant<float, RecF, 2, 2, 128, 3, 2>(B_, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 18: return launch_variant<double, RecD, 2, 1, 128, 3, 2>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 19: return launch_variant<double, RecD, 3, 1, 128, 2, 2>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 20: return launch_variant<double, RecD, 2, 2, 128, 1, 2>(B_, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    default: return fail(kErrInvalid, "bad nbody variant");
  }

}

}  // namespace uvlm

namespace uvlm {

// FP32 batch tiles the batch autotuner chooses from: column-bounded packed
// FP32x2 walkers with the far-field walker, H node rows per strip.
constexpr int kBatchTileH[kNumBatchTilesF] = {3, 2, 4};

int nbody_batch_rows(NBodyPrec prec, bool padded) {
  (void)padded;  // one FP32 class: the column-bounded packed tile takes every sheet
  return prec == kNBodyFP32 ? kBatchHFP : kBatchHD;
}

const char* nbody_batch_tile_name(NBodyPrec prec, int tile) {
  static const char* names[kNumBatchTilesF] = {"fp32_h3_t2_b128_x2f", "fp32_h2_t2_b128_x2f", "fp32_h4_t2_b128_x2f"};
  if (prec != kNBodyFP32) return "fp64_h2_t1_b128";
  return (tile >= 0 && tile < kNumBatchTilesF) ? names[tile] : "?";
}

long long nbody_batch_partial_doubles(NBodyPrec prec, const NBodyBatchInput* in, int n) {
  // the bound of every tile the batch may run (the fewest rows per strip
  // make the most strips, hence the most source splits)
  long long worst = 0;
  const int tiles = prec == kNBodyFP32 ? kNumBatchTilesF : 1;
  for (int t = 0; t < tiles; ++t) {
    const int H = prec == kNBodyFP32 ? kBatchTileH[t] : kBatchHD;
    long long total = 0;
    for (int c = 0; c < n; ++c) {
      Blocks B{};
      const long long strips = fill_blocks(B, in[c].blocks, in[c].n_blocks, H);
      const long long splits = (strips + kBatchStripsPerItem - 1) / kBatchStripsPerItem;
      total += splits * 3 * in[c].n_tgt;
    }
    worst = std::max(worst, total);
  }
  return worst;
}

namespace {
template <class T, class Rec, int H, int TPT, bool PAD, int PK>
int batch_grid_of(int num_sms) {
  const void* k = (const void*)batch_nbody_kernel<T, Rec, H, TPT, kBatchBlock, kBatchMinB, PAD, PK>;
  const size_t smem = strip_smem<Rec, H, kBatchBlock, PK>();
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, kBatchBlock, smem) != cudaSuccess || occ < 1) occ = 1;
  return num_sms * occ;
}

template <int H>
Error batch_eval_f32(const NBodyBatchInput* d_in, int n, const double* tx, const double* ty, const double* tz,
                     const RecF* rf, double* partial, long long partial_cap, NBodyBatchPlan* d_plan,
                     long long* d_totals, int* status, int grid, cudaStream_t st) {
  batch_plan_kernel<H, kBatchBlock * kBatchTptF><<<1, 256, 0, st>>>(d_in, n, -1, d_plan, partial_cap, d_totals,
                                                                    status);
  UVLM_LAUNCH_CHECK();
  batch_nbody_kernel<float, RecF, H, kBatchTptF, kBatchBlock, kBatchMinB, true, kBatchPadPK>
      <<<grid, kBatchBlock, strip_smem<RecF, H, kBatchBlock, kBatchPadPK>(), st>>>(d_plan, n, d_totals, tx, ty, tz,
                                                                                 rf, partial);
  UVLM_LAUNCH_CHECK();
  return ok();
}
}  // namespace

NBodyBatchGrids nbody_batch_grids(NBodyPrec prec, int num_sms) {
  NBodyBatchGrids g;
  if (prec == kNBodyFP32) {
    g.general = 0;
    g.tiles[0] = batch_grid_of<float, RecF, 3, kBatchTptF, true, kBatchPadPK>(num_sms);
    g.tiles[1] = batch_grid_of<float, RecF, 2, kBatchTptF, true, kBatchPadPK>(num_sms);
    g.tiles[2] = batch_grid_of<float, RecF, 4, kBatchTptF, true, kBatchPadPK>(num_sms);
    g.padded = g.tiles[0];
  } else {
    g.general = batch_grid_of<double, RecD, kBatchHD, kBatchTptD, false, 0>(num_sms);
  }
  return g;
}

Error nbody_batch_eval(NBodyPrec prec, const NBodyBatchInput* d_in, int n, const double* tx, const double* ty,
                       const double* tz, double* vx, double* vy, double* vz, const void* records, double* partial,
                       long long partial_cap, NBodyBatchPlan* d_plan, long long* d_totals, int* status,
                       const NBodyBatchGrids& grids, cudaStream_t st) {
  if (n <= 0) return ok();
  auto reduce = [&](int grid) -> Error {
    batch_reduce_kernel<<<grid, 256, 0, st>>>(d_plan, n, d_totals, partial, vx, vy, vz);
    UVLM_LAUNCH_CHECK();
    return ok();
  };
  if (prec == kNBodyFP32) {
    // every problem: the column-bounded packed FP32x2 tile with the far-field
    // walker, in the height the batch's autotuner chose
    const RecF* rf = reinterpret_cast<const RecF*>(records);
    const int t = (grids.tile >= 0 && grids.tile < kNumBatchTilesF) ? grids.tile : 0;
    const int grid = grids.tiles[t];
    switch (t) {
      case 1: UVLM_TRY(batch_eval_f32<2>(d_in, n, tx, ty, tz, rf, partial, partial_cap, d_plan, d_totals, status, grid, st)); break;
      case 2: UVLM_TRY(batch_eval_f32<4>(d_in, n, tx, ty, tz, rf, partial, partial_cap, d_plan, d_totals, status, grid, st)); break;
      default: UVLM_TRY(batch_eval_f32<3>(d_in, n, tx, ty, tz, rf, partial, partial_cap, d_plan, d_totals, status, grid, st)); break;
    }
    return reduce(grid);
  }
  batch_plan_kernel<kBatchHD, kBatchBlock * kBatchTptD><<<1, 256, 0, st>>>(d_in, n, -1, d_plan, partial_cap,
                                                                           d_totals, status);
  UVLM_LAUNCH_CHECK();
  batch_nbody_kernel<double, RecD, kBatchHD, kBatchTptD, kBatchBlock, kBatchMinB, false, 0>
      <<<grids.general, kBatchBlock, strip_smem<RecD, kBatchHD, kBatchBlock, 0>(), st>>>(
          d_plan, n, d_totals, tx, ty, tz, reinterpret_cast<const RecD*>(records), partial);
  UVLM_LAUNCH_CHECK();
  return reduce(grids.general);
}

}  // namespace uvlm
