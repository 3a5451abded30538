// nbody.cu -- strip-tiled Biot-Savart N-body (FP32 hi/lo and FP64 forms).
#include "nbody.cuh"
#include "bs_math.cuh"

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
    Rec r;
    if constexpr (sizeof(Rec) == sizeof(RecF)) {
      const float hx = (float)p[0], hy = (float)p[1], hz = (float)p[2];
      r.hi = make_float4(hx, hy, hz, (float)(gS * s));
      r.lo = make_float4((float)(p[0] - (double)hx), (float)(p[1] - (double)hy),
                         (float)(p[2] - (double)hz), (float)(gH * s));
    } else {
      r.a = make_double4(p[0], p[1], p[2], gS * s);
      r.b = make_double2(gH * s, 0.0);
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

template <class T, class Rec>
__device__ __forceinline__ Node<T> node_from(const Rec& r, const Tgt<T>& t) {
  if constexpr (sizeof(T) == 4) {
    const float x = (t.hx - r.hi.x) + (t.lx - r.lo.x);
    const float y = (t.hy - r.hi.y) + (t.ly - r.lo.y);
    const float z = (t.hz - r.hi.z) + (t.lz - r.lo.z);
    return make_node<float>(x, y, z);
  } else {
    return make_node<double>(t.hx - r.a.x, t.hy - r.a.y, t.hz - r.a.z);
  }
}
template <class T, class Rec>
__device__ __forceinline__ void strengths(const Rec& r, T& gS, T& gH) {
  if constexpr (sizeof(T) == 4) {
    gS = r.hi.w;
    gH = r.lo.w;
  } else {
    gS = r.a.w;
    gH = r.b.x;
  }
}

// Walk one staged strip for TPT targets.
template <class T, class Rec, int H, int TPT>
__device__ __forceinline__ void walk_strip(const Rec* sm, const StripInfo& si, const Tgt<T> (&tg)[TPT],
                                           T (&acc)[TPT][3]) {
  Node<T> prev[TPT][H];
  T pgS[H];
#pragma unroll
  for (int r = 0; r < H; ++r) pgS[r] = (T)0;
  const int nr = si.nr, n_rows = si.n_rows, n_cols = si.n_cols;
  for (int j = 0; j < n_cols; ++j) {
    Node<T> cur[TPT][H + 1];
    T gS[H], gH[H];
#pragma unroll
    for (int r = 0; r <= H; ++r) {
      if (r < nr) {
        const Rec rec = sm[r * n_cols + j];
        if (r < H) strengths<T, Rec>(rec, gS[r], gH[r]);
#pragma unroll
        for (int q = 0; q < TPT; ++q) cur[q][r] = node_from<T, Rec>(rec, tg[q]);
      }
    }
    const bool col_h = (j < n_cols - 1) || si.last_h;
#pragma unroll
    for (int r = 0; r < H; ++r) {
      if (r < n_rows && r + 1 < nr && col_h) {
#pragma unroll
        for (int q = 0; q < TPT; ++q) segment<T>(cur[q][r], cur[q][r + 1], gH[r], acc[q][0], acc[q][1], acc[q][2]);
      }
    }
    if (j > 0) {
#pragma unroll
      for (int r = 0; r < H; ++r) {
        if (r < n_rows) {
#pragma unroll
          for (int q = 0; q < TPT; ++q) segment<T>(prev[q][r], cur[q][r], pgS[r], acc[q][0], acc[q][1], acc[q][2]);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < H; ++r) {
      if (r < n_rows) {
        pgS[r] = gS[r];
#pragma unroll
        for (int q = 0; q < TPT; ++q) prev[q][r] = cur[q][r];
      }
    }
  }
}

template <class T, class Rec, int H, int TPT, int BLOCK>
__global__ void __launch_bounds__(BLOCK) nbody_kernel(Blocks B, long long n_strips, long long strips_per_split,
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
  int H, TPT, BLOCK;
};

constexpr Variant kVariants[] = {
    {"fp64_h4_t1_b128", kNBodyFP64, 4, 1, 128},
    {"fp64_h2_t1_b256", kNBodyFP64, 2, 1, 256},
    {"fp32_h4_t1_b256", kNBodyFP32, 4, 1, 256},
    {"fp32_h4_t2_b128", kNBodyFP32, 4, 2, 128},
    {"fp32_h2_t2_b128", kNBodyFP32, 2, 2, 128},
};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

template <class T, class Rec, int H, int TPT, int BLOCK>
Error launch_variant(const Blocks& B, long long n_strips, const double* tx, const double* ty, const double* tz,
                     long long n_targets, const Rec* rec, NBodyWork* work, double* vx, double* vy, double* vz,
                     int num_sms, cudaStream_t st) {
  auto kern = nbody_kernel<T, Rec, H, TPT, BLOCK>;
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
  switch (variant) {
    case 0: return launch_variant<double, RecD, 4, 1, 128>(B, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 1: return launch_variant<double, RecD, 2, 1, 256>(B, strips, tx, ty, tz, n_targets, rd, work, vx, vy, vz, num_sms, st);
    case 2: return launch_variant<float, RecF, 4, 1, 256>(B, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 3: return launch_variant<float, RecF, 4, 2, 128>(B, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    case 4: return launch_variant<float, RecF, 2, 2, 128>(B, strips, tx, ty, tz, n_targets, rf, work, vx, vy, vz, num_sms, st);
    default: return fail(kErrInvalid, "bad nbody variant");
  }
}

}  // namespace uvlm
