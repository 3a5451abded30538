// nbody.cu -- strip-tiled Biot-Savart N-body (FP32 hi/lo and FP64 forms).
#include "nbody.cuh"

namespace uvlm {
namespace {

// ------------------------------------------------------------ record build
__device__ inline double ring_gamma(const SheetView& v, int n, int i, int j) {
  const int R = v.node_rows - 1;
  if (i < 0 || i >= R || j < 0 || j >= v.cols) return 0.0;
  return v.gamma[((long long)n * v.g_rows_alloc + v.g_row0 + i) * v.cols + j];
}

template <class Rec>
__global__ void build_records_kernel(SheetView v, Rec* out) {
  const long long total = (long long)v.num * v.node_rows * (v.cols + 1);
  const double s = 1.0 / (4.0 * kPi);
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
       k += (long long)gridDim.x * blockDim.x) {
    const int C1 = v.cols + 1;
    const int j = (int)(k % C1);
    const long long nr = k / C1;
    const int i = (int)(nr % v.node_rows);
    const int n = (int)(nr / v.node_rows);
    const double* p = v.pos + (((long long)n * v.rows_alloc + v.row0 + i) * C1 + j) * 3;
    const int R = v.node_rows - 1;
    // strengths: spanwise S(i,j) and chordwise H(i,j) (nbody.cuh)
    const double gS = (j < v.cols) ? ring_gamma(v, n, i, j) - ring_gamma(v, n, i - 1, j) : 0.0;
    const double gH = (i < R && !v.spanwise_only) ? ring_gamma(v, n, i, j - 1) - ring_gamma(v, n, i, j) : 0.0;
    // segment vectors s0 = p(i,j+1) - p(i,j), h0 = p(i+1,j) - p(i,j)
    double s0[3] = {0, 0, 0}, h0[3] = {0, 0, 0};
    if (j < v.cols)
      for (int d = 0; d < 3; ++d) s0[d] = p[3 + d] - p[d];
    if (i < R)
      for (int d = 0; d < 3; ++d) h0[d] = p[3 * C1 + d] - p[d];
    Rec r;
    if constexpr (sizeof(Rec) == sizeof(RecF)) {
      const float hx = (float)p[0], hy = (float)p[1], hz = (float)p[2];
      r.hi = make_float4(hx, hy, hz, (float)(gS * s));
      r.lo = make_float4((float)(p[0] - (double)hx), (float)(p[1] - (double)hy),
                         (float)(p[2] - (double)hz), (float)(gH * s));
      r.sv = make_float4((float)s0[0], (float)s0[1], (float)s0[2], (float)h0[0]);
      r.hv = make_float4((float)h0[1], (float)h0[2], 0.f, 0.f);
    } else {
      r.a = make_double4(p[0], p[1], p[2], gS * s);
      r.b = make_double4(gH * s, s0[0], s0[1], s0[2]);
      r.c = make_double4(h0[0], h0[1], h0[2], 0.0);
    }
    out[k] = r;
  }
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

struct Blocks {
  SourceBlock b[4];
  int n;
  int strips_per_sheet[4];
  int chunks[4];
  long long strip_begin[5];
};

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

template <class T>
struct Tgt {
  T hx, hy, hz;  // FP32: hi part; FP64: the position
  T lx, ly, lz;  // FP32: lo part; FP64: unused
};

template <class T>
struct NodeV {
  T rx, ry, rz;  // x - p
  T ux, uy, uz;  // (x - p)/|x - p|  (NaN/inf lanes when x == p are cut by |d|^2)
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
    const float inv = nb_rsqrt(n.rx * n.rx + n.ry * n.ry + n.rz * n.rz);
    n.ux = n.rx * inv;
    n.uy = n.ry * inv;
    n.uz = n.rz * inv;
  } else {
    n.rx = t.hx - r.a.x;
    n.ry = t.hy - r.a.y;
    n.rz = t.hz - r.a.z;
    const double inv = rsqrt(n.rx * n.rx + n.ry * n.ry + n.rz * n.rz);
    n.ux = n.rx * inv;
    n.uy = n.ry * inv;
    n.uz = n.rz * inv;
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

// Segment start=A -> end=B at x (src/vortex.cpp:24-38): r0 = B - A, r1 = x - A,
// d = r0 x r1 (= r1 x r2), K = g r0.(u1 - u2) / |d|^2, cut when |d|^2 < 1e-10.
// |x - A| < 1e-10 or |x - B| < 1e-10 implies |d|^2 < 1e-10 for |x - p| < 1e5,
// so the reference's node cut-off is contained in the |d|^2 test (and the
// select also discards the NaN that rsqrt(0) produces in u).
template <class T>
__device__ __forceinline__ void seg(const SegV<T>& r0, const NodeV<T>& a, const NodeV<T>& b, T g, T& vx, T& vy,
                                    T& vz) {
  const T dx = r0.y * a.rz - r0.z * a.ry;
  const T dy = r0.z * a.rx - r0.x * a.rz;
  const T dz = r0.x * a.ry - r0.y * a.rx;
  const T d2 = dx * dx + dy * dy + dz * dz;
  const T dot = r0.x * (a.ux - b.ux) + r0.y * (a.uy - b.uy) + r0.z * (a.uz - b.uz);
  T k;
  if constexpr (sizeof(T) == 4) {
    k = g * dot * nb_rcp(d2);
  } else {
    k = g * dot * __drcp_rn(d2);
  }
  k = (d2 < (T)kCutD2) ? (T)0 : k;
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

template <class T, class Rec, int H, int TPT, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) nbody_kernel(Blocks B, long long n_strips, long long strips_per_split,
                                                       const double* __restrict__ tx, const double* __restrict__ ty,
                                                       const double* __restrict__ tz, long long n_targets,
                                                       const Rec* __restrict__ rec, double* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Rec* buf0 = reinterpret_cast<Rec*>(smem_raw);
  Rec* buf1 = buf0 + (H + 1) * (kStripCols + 1);

  const long long tile0 = (long long)blockIdx.x * BLOCK * TPT;
  Tgt<T> tg[TPT];
  double accd[TPT][3];
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    long long t = tile0 + threadIdx.x + (long long)q * BLOCK;
    if (t >= n_targets) t = n_targets - 1;  // padded lanes recompute the last target
    const double x = tx[t], y = ty[t], z = tz[t];
    if constexpr (sizeof(T) == 4) {
      tg[q].hx = (float)x; tg[q].hy = (float)y; tg[q].hz = (float)z;
      tg[q].lx = (float)(x - (double)tg[q].hx);
      tg[q].ly = (float)(y - (double)tg[q].hy);
      tg[q].lz = (float)(z - (double)tg[q].hz);
    } else {
      tg[q].hx = x; tg[q].hy = y; tg[q].hz = z;
      tg[q].lx = tg[q].ly = tg[q].lz = 0;
    }
    accd[q][0] = accd[q][1] = accd[q][2] = 0.0;
  }

  const long long s_begin = (long long)blockIdx.y * strips_per_split;
  const long long s_end = min(n_strips, s_begin + strips_per_split);
  if (s_begin < s_end) {
    StripInfo si = decode_strip<H>(B, s_begin);
    stage_strip<Rec>(buf0, rec, si);
    for (long long s = s_begin; s < s_end; ++s) {
      Rec* cur = ((s - s_begin) & 1) ? buf1 : buf0;
      Rec* nxt = ((s - s_begin) & 1) ? buf0 : buf1;
      StripInfo sn;
      const bool has_next = s + 1 < s_end;
      if (has_next) {
        sn = decode_strip<H>(B, s + 1);
        stage_strip<Rec>(nxt, rec, sn);
        asm volatile("cp.async.wait_group 1;");
      } else {
        asm volatile("cp.async.wait_group 0;");
      }
      __syncthreads();
      T acc[TPT][3];
#pragma unroll
      for (int q = 0; q < TPT; ++q) acc[q][0] = acc[q][1] = acc[q][2] = (T)0;
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
};

// Tile shapes: H owned node rows per strip, TPT targets per thread, BLOCK
// threads, MINB resident CTAs per SM requested from the register allocator.
constexpr Variant kVariants[] = {
    {"fp64_h4_t1_b128", kNBodyFP64, 4, 1, 128, 1},
    {"fp64_h2_t1_b256", kNBodyFP64, 2, 1, 256, 1},
    {"fp32_h4_t1_b256", kNBodyFP32, 4, 1, 256, 2},
    {"fp32_h4_t2_b128", kNBodyFP32, 4, 2, 128, 3},
    {"fp32_h2_t2_b128", kNBodyFP32, 2, 2, 128, 3},
    {"fp32_h4_t1_b128_m4", kNBodyFP32, 4, 1, 128, 4},
    {"fp32_h3_t2_b128_m4", kNBodyFP32, 3, 2, 128, 4},
    {"fp32_h2_t1_b256_m3", kNBodyFP32, 2, 1, 256, 3},
    {"fp64_h2_t2_b128", kNBodyFP64, 2, 2, 128, 1},
    {"fp64_h2_t1_b128_m3", kNBodyFP64, 2, 1, 128, 3},
    {"fp64_h2_t1_b256_m2", kNBodyFP64, 2, 1, 256, 2},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

template <class T, class Rec, int H, int TPT, int BLOCK, int MINB>
Error launch_variant(const Blocks& B, long long n_strips, const double* tx, const double* ty, const double* tz,
                     long long n_targets, const Rec* rec, NBodyWork* work, double* vx, double* vy, double* vz,
                     int num_sms, cudaStream_t st) {
  auto kern = nbody_kernel<T, Rec, H, TPT, BLOCK, MINB>;
  const size_t smem = 2 * sizeof(Rec) * (H + 1) * (kStripCols + 1);
  static bool attr_done = false;
  if (!attr_done) {
    UVLM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_done = true;
  }
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
  if (splits < 1) splits = 1;
  const long long sps = (n_strips + splits - 1) / splits;
  splits = (n_strips + sps - 1) / sps;
  const long long need = splits * 3 * n_targets;
  if (work->partial_cap < need) return fail(kErrCapacity, "nbody partial buffer too small");
  dim3 grid((unsigned)tiles, (unsigned)splits);
  kern<<<grid, BLOCK, smem, st>>>(B, n_strips, sps, tx, ty, tz, n_targets, rec, work->partial);
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
  B.n = 0;
  long long strips = 0;
  for (int i = 0; i < n_blocks && B.n < 4; ++i) {
    const SourceBlock& sb = blocks[i];
    if (sb.num <= 0 || sb.node_rows < 2 || sb.cols <= 0) continue;  // no rings -> no segments
    B.b[B.n] = sb;
    const int groups = (sb.node_rows + V.H - 1) / V.H;
    const int chunks = (sb.cols + kStripCols - 1) / kStripCols;
    B.chunks[B.n] = chunks;
    B.strips_per_sheet[B.n] = groups * chunks;
    B.strip_begin[B.n] = strips;
    strips += (long long)sb.num * groups * chunks;
    B.n++;
  }
  B.strip_begin[B.n] = strips;
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
    default: return fail(kErrInvalid, "bad nbody variant");
  }

}

}  // namespace uvlm
