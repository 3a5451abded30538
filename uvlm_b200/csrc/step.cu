// step.cu -- kinematics, shedding, geometry, assembly, RHS, loads, advection.
#include "bs_math.cuh"
#include "step.cuh"
#include "step_math.cuh"

namespace uvlm {
namespace {

__global__ void kinematics_kernel(const uvlm_kinematics* __restrict__ kin, WingShape ws, const double* pos_init,
                                  double* pos, double t) {
  const long long per = (long long)(ws.R + 1) * (ws.C + 1);
  const long long total = per * ws.num;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(k / per);
    st3(pos + 3 * k, perfome(kin[n], ld3(pos_init + 3 * k), t));
  }
}

// SimpleSimulator::Shed (simple_simulator.cpp:171-188): prepend the TE node
// row; from step 1 on also the TE circulation row of the previous solve.
__global__ void shed_kernel(WingShape ws, const double* wing_pos, const double* wing_gamma, WakeLayout wl,
                            double* wake_pos, double* wake_gamma, int shed_gamma) {
  const int C1 = ws.C + 1;
  const int total = ws.num * C1;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    const int n = k / C1, j = k % C1;
    const double* p = wing_pos + 3 * ws.node(n, ws.R, j);
    double* q = wake_pos + 3 * wl.node(n, 0, j);
    q[0] = p[0];
    q[1] = p[1];
    q[2] = p[2];
    if (shed_gamma && j < ws.C) wake_gamma[wl.ring(n, 0, j)] = wing_gamma[ws.ring(n, ws.R - 1, j)];
  }
}

__global__ void panel_geometry_kernel(const uvlm_kinematics* __restrict__ kin, WingShape ws, const double* pos,
                                      const double* pos_init, double t, double* cx, double* cy, double* cz,
                                      double* normal, double* area, double* uls) {
  const int per = ws.R * ws.C;
  const int total = per * ws.num;
  for (int K = blockIdx.x * blockDim.x + threadIdx.x; K < total; K += gridDim.x * blockDim.x) {
    const int n = K / per, i = (K % per) / ws.C, j = K % ws.C;
    const d3 p00 = ld3(pos + 3 * ws.node(n, i, j)), p10 = ld3(pos + 3 * ws.node(n, i + 1, j));
    const d3 p11 = ld3(pos + 3 * ws.node(n, i + 1, j + 1)), p01 = ld3(pos + 3 * ws.node(n, i, j + 1));
    // CollocationPoints (simple_simulator.cpp:19-32)
    const d3 c = dvs(add(add(add(p00, p10), p11), p01), 4);
    cx[K] = c.x;
    cy[K] = c.y;
    cz[K] = c.z;
    // Normals (:34-50)
    st3(normal + 3 * K, normalized(cross(sub(p11, p00), sub(p01, p10))));
    // CalcPanelArea (src/calc_load/joukowski.cpp:55-67)
    area[K] = norm(cross(sub(p10, p00), sub(p01, p00)));
    const d3 q00 = ld3(pos_init + 3 * ws.node(n, i, j)), q10 = ld3(pos_init + 3 * ws.node(n, i + 1, j));
    const d3 q11 = ld3(pos_init + 3 * ws.node(n, i + 1, j + 1)), q01 = ld3(pos_init + 3 * ws.node(n, i, j + 1));
    const d3 c0 = dvs(add(add(add(q00, q10), q11), q01), 4);
    st3(uls + 3 * K, morph_velocity(kin[n], c0, t));
  }
}

// ---------------------------------------------------------------- assembly
// A[K][L] = VORING(c_K, L, 1) . n_K by unique lattice segments.  Ring (i, j)
// is p0 -> p1 -> p2 -> p3 -> p0 with p0 = (i, j), p1 = (i, j+1), p2 = (i+1, j+1),
// p3 = (i+1, j) (src/vortex.cpp:145-160): the spanwise segment S(i, j) =
// (i, j) -> (i, j+1), the chordwise H(i, j+1) = (i, j+1) -> (i+1, j+1), then
// S(i+1, j) and H(i, j) backwards.  Neighbouring rings share those segments
// with opposite signs, so one lane per (collocation point K, node column j of
// wing n) walks the node rows i = 0..R, forms the nodes (i, j) and (i, j+1)
// once per row and the segments S(i, j) and H(i-1, j) once, takes H(i-1, j+1)
// from the next lane, and writes ring (i-1, j) = S(i-1, j) + H(i-1, j+1) -
// S(i, j) - H(i-1, j): two segment evaluations per (point, ring) pair instead
// of four, two nodes instead of four.  Lanes run over (K, node column) with 31
// new positions per warp, so lane 31 only supplies its chordwise segment to
// lane 30; node column C of a wing (no ring of its own) does the same for
// column C - 1.  The segment arithmetic is the ring form's (bs_math.cuh); a
// backward segment is the negated forward one, equal to rounding.
constexpr int kAsmBlock = 128;
constexpr int kAsmPerWarp = 31;

template <class T, class OutT>
__global__ void __launch_bounds__(kAsmBlock) assemble_kernel(WingShape ws, const double* __restrict__ pos,
                                                             const double* __restrict__ cx, const double* __restrict__ cy,
                                                             const double* __restrict__ cz,
                                                             const double* __restrict__ normal, OutT* A) {
  const int C1 = ws.C + 1;
  const int NC = ws.num * C1;
  const int N = ws.num * ws.R * ws.C;
  const long long P = (long long)N * NC;
  const int lane = threadIdx.x & 31;
  const long long p0 = ((long long)blockIdx.x * (kAsmBlock / 32) + (threadIdx.x >> 5)) * kAsmPerWarp;
  if (p0 >= P) return;  // the whole warp
  const long long p = min(p0 + lane, P - 1);
  const int K = (int)(p / NC);
  const int jn = (int)(p - (long long)K * NC);
  const int n = jn / C1, j = jn - n * C1;
  const bool owner = lane < kAsmPerWarp && p0 + lane < P && j < ws.C;
  const int j1 = min(j + 1, ws.C);
  const double X = cx[K], Y = cy[K], Z = cz[K];
  const T hx = (T)X, hy = (T)Y, hz = (T)Z;
  const T lx = (T)(X - (double)hx), ly = (T)(Y - (double)hy), lz = (T)(Z - (double)hz);
  const T nx = (T)normal[3 * K], ny = (T)normal[3 * K + 1], nz = (T)normal[3 * K + 2];
  const T g = (T)(1.0 / (4.0 * kPi));
  // x - p from the hi/lo parts of both (FP64: lo = 0, the plain difference)
  auto node_at = [&](int i, int jj) {
    const double* q = pos + 3 * ws.node(n, i, jj);
    const double qx = q[0], qy = q[1], qz = q[2];
    const T px = (T)qx, py = (T)qy, pz = (T)qz;
    return make_node<T>((hx - px) + (lx - (T)(qx - (double)px)), (hy - py) + (ly - (T)(qy - (double)py)),
                        (hz - pz) + (lz - (T)(qz - (double)pz)));
  };
  Node<T> a = node_at(0, j), b = node_at(0, j1);
  T sx = 0, sy = 0, sz = 0;  // S(i-1, j)
  segment<T>(a, b, g, sx, sy, sz);
  OutT* row = A + (long long)K * N + ws.ring(n, 0, j);
  for (int i = 1; i <= ws.R; ++i) {
    const Node<T> a2 = node_at(i, j), b2 = node_at(i, j1);
    T hvx = 0, hvy = 0, hvz = 0;  // H(i-1, j)
    segment<T>(a, a2, g, hvx, hvy, hvz);
    const T hnx = __shfl_down_sync(0xffffffffu, hvx, 1);  // H(i-1, j+1)
    const T hny = __shfl_down_sync(0xffffffffu, hvy, 1);
    const T hnz = __shfl_down_sync(0xffffffffu, hvz, 1);
    T s2x = 0, s2y = 0, s2z = 0;  // S(i, j)
    segment<T>(a2, b2, g, s2x, s2y, s2z);
    if (owner) {
      const T vx = ((sx + hnx) - s2x) - hvx;
      const T vy = ((sy + hny) - s2y) - hvy;
      const T vz = ((sz + hnz) - s2z) - hvz;
      row[(long long)(i - 1) * ws.C] = (OutT)(vx * nx + vy * ny + vz * nz);
    }
    a = a2;
    b = b2;
    sx = s2x;
    sy = s2y;
    sz = s2z;
  }
}

// Legacy AoS assembly (src/linear.inl:14-32): A[i][j] = ring_j.BiotSavartLaw(
// centroid_i, 1).Normal_i with ForEachSegment order nodes[k+1] -> nodes[k].
__global__ void ring_geometry_kernel(const double* rings, int n, double* centroid, double* normal) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double* r = rings + 12 * i;
    const d3 a = ld3(r), b = ld3(r + 3), c = ld3(r + 6), d = ld3(r + 9);
    st3(centroid + 3 * i, dvs(add(add(add(a, b), c), d), 4));                 // vortex.cpp:98-100
    st3(normal + 3 * i, normalized(cross(sub(b, d), sub(c, a))));               // vortex.cpp:82-87
  }
}

__global__ void assemble_rings_kernel(const double* rings, int n, const double* centroid, const double* normal,
                                      double* A) {
  const long long total = (long long)n * n;
  const double g = 1.0 / (4.0 * kPi);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / n), j = (int)(q % n);
    const d3 x = ld3(centroid + 3 * i);
    const double* r = rings + 12 * j;
    Node<double> nd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) nd[k] = make_node<double>(x.x - r[3 * k], x.y - r[3 * k + 1], x.z - r[3 * k + 2]);
    double vx = 0, vy = 0, vz = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) segment<double>(nd[(k + 1) & 3], nd[k], g, vx, vy, vz);
    A[q] = vx * normal[3 * i] + vy * normal[3 * i + 1] + vz * normal[3 * i + 2];
  }
}

__global__ void legacy_rhs_kernel(const uvlm_kinematics* __restrict__ kin, const int* __restrict__ kin_of,
                                  const double* rings0, int n, const double* normal, d3 fs, double t,
                                  const double* wake_vel, double* b) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double* r = rings0 + 12 * i;
    const d3 c0 = dvs(add(add(add(ld3(r), ld3(r + 3)), ld3(r + 6)), ld3(r + 9)), 4);  // ReferenceCentroid
    const d3 nl = ld3(normal + 3 * i);
    double v = dot(morph_velocity(kin[kin_of ? kin_of[i] : 0], c0, t), nl) - dot(fs, nl);
    if (wake_vel) v -= dot(ld3(wake_vel + 3 * i), nl);
    b[i] = v;
  }
}

__global__ void rhs_kernel(int N, const double* uwx, const double* uwy, const double* uwz, const double* uls,
                           const double* normal, d3 ff, double* b) {
  for (int K = blockIdx.x * blockDim.x + threadIdx.x; K < N; K += gridDim.x * blockDim.x) {
    const d3 uw = mk(uwx ? uwx[K] : 0.0, uwy ? uwy[K] : 0.0, uwz ? uwz[K] : 0.0);
    const d3 u = sub(uw, add(ld3(uls + 3 * K), ff));
    b[K] = -dot(u, ld3(normal + 3 * K));
  }
}

__global__ void line_prep_kernel(const uvlm_kinematics* __restrict__ kin, WingShape ws, const double* pos,
                                 const double* pos_init, double t, double* tx, double* ty, double* tz,
                                 double* line_uls) {
  const int Lw = ws.lines_per_wing();
  const int total = Lw * ws.num;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
    const int n = k / Lw, q = k % Lw;
    long long a, b;
    line_nodes(ws, n, q, a, b);
    const d3 mp = dvs(add(ld3(pos + 3 * a), ld3(pos + 3 * b)), 2);
    const d3 mp0 = dvs(add(ld3(pos_init + 3 * a), ld3(pos_init + 3 * b)), 2);
    tx[k] = mp.x;
    ty[k] = mp.y;
    tz[k] = mp.z;
    st3(line_uls + 3 * k, morph_velocity(kin[n], mp0, t));
  }
}

template <int BS>
__device__ inline double block_sum(double v, double* sh) {
  for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  v = (threadIdx.x < BS / 32) ? sh[threadIdx.x] : 0.0;
  if (wid == 0)
    for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  return v;  // valid in thread 0
}

// CalcLoad (simple_simulator.cpp:195-233): JoukowskiSteady over the lines
// (U x dl) * Gamma with U = (-ff + Ub + Uw)(mid) - Uls(mid0), plus
// JoukowskiUnsteady n * dGamma/dt * A; C = F / (0.5 |ff|^2 chord span).
template <int BS>
__global__ void __launch_bounds__(BS) loads_kernel(WingShape ws, const double* pos, const double* gamma,
                                                    const double* gamma_prev, const double* normal,
                                                    const double* area, const double* vx, const double* vy,
                                                    const double* vz, const double* line_uls, d3 ff,
                                                    const double* chord_span, double t, double dt, double* row) {
  __shared__ double sh[32];
  const int n = blockIdx.x;
  const int Lw = ws.lines_per_wing();
  double f[3] = {0, 0, 0}, u[3] = {0, 0, 0};
  for (int q = threadIdx.x; q < Lw; q += BS) {
    const int k = n * Lw + q;
    long long a, b;
    line_nodes(ws, n, q, a, b);
    const d3 dl = sub(ld3(pos + 3 * b), ld3(pos + 3 * a));
    const d3 U = sub(add(mk(-ff.x, -ff.y, -ff.z), mk(vx[k], vy[k], vz[k])), ld3(line_uls + 3 * k));
    const d3 df = scl(cross(U, dl), line_strength(ws, gamma, n, q));
    f[0] += df.x;
    f[1] += df.y;
    f[2] += df.z;
  }
  const int per = ws.R * ws.C;
  for (int p = threadIdx.x; p < per; p += BS) {
    const int K = n * per + p;
    const double dgdt = (gamma[K] - gamma_prev[K]) / dt;
    const d3 df = scl(scl(ld3(normal + 3 * K), dgdt), area[K]);
    u[0] += df.x;
    u[1] += df.y;
    u[2] += df.z;
  }
  double F[3];
  for (int d = 0; d < 3; ++d) {
    const double fs = block_sum<BS>(f[d], sh);
    const double fu = block_sum<BS>(u[d], sh);
    F[d] = fs + fu;
  }
  if (threadIdx.x == 0) {
    const double Q = norm(ff);
    const double S = chord_span[2 * n] * chord_span[2 * n + 1];
    const double den = 0.5 * Q * Q * S;
    if (n == 0) row[0] = t;
    row[1 + 2 * n] = F[0] / den;
    row[2 + 2 * n] = F[2] / den;
  }
}

// Wake nodes of rows first_row.. of every wake sheet as SoA targets.
__global__ void gather_wake_kernel(WakeLayout wl, const double* pos, int first_row, double* tx, double* ty,
                                   double* tz) {
  const int C1 = wl.C + 1;
  const int rows = wl.node_rows - first_row;
  const long long total = (long long)wl.num * rows * C1;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(k % C1);
    const long long nr = k / C1;
    const int i = (int)(nr % rows) + first_row, n = (int)(nr / rows);
    const double* p = pos + 3 * wl.node(n, i, j);
    tx[k] = p[0];
    ty[k] = p[1];
    tz[k] = p[2];
  }
}

// vx/vy/vz hold the induced velocities of the wake rows vrow0.. (the gather's
// first_row); rows above vrow0 take -ff alone where the mode reads them.
__global__ void advect_kernel(int mode, WakeLayout wl, double* x, double* pos2, double* k1, double* k2, double* k3,
                              double* vprev, int has_vprev, const double* vx, const double* vy, const double* vz,
                              d3 ff, double dt, int ignore, int vrow0) {
  const int C1 = wl.C + 1;
  const long long total = (long long)wl.num * wl.node_rows * C1;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(k % C1);
    const long long nr = k / C1;
    const int i = (int)(nr % wl.node_rows), n = (int)(nr / wl.node_rows);
    const long long P = 3 * wl.node(n, i, j);
    const d3 mff = mk(-ff.x, -ff.y, -ff.z);
    d3 u = mff;
    if (i >= vrow0) {
      const long long ti = ((long long)n * (wl.node_rows - vrow0) + (i - vrow0)) * C1 + j;
      u = add(mff, mk(vx[ti], vy[ti], vz[ti]));
    }
    const d3 xp = ld3(x + P);
    switch (mode) {
      case kAdvEuler:  // src/advect.cpp:11-22
        st3(x + P, add(xp, scl(u, dt)));
        break;
      case kAdvRK2K1:  // src/advect.cpp:40-57
        st3(k1 + P, u);
        st3(pos2 + P, add(xp, scl(u, dt)));
        break;
      case kAdvRK2Upd: {  // src/advect.cpp:71-79
        const d3 a = ld3(k1 + P);
        st3(x + P, i > ignore ? add(xp, dvs(scl(add(a, u), dt), 2)) : add(xp, scl(a, dt)));
        break;
      }
      case kAdvRK4K1:  // src/advect.cpp:98-118
        st3(k1 + P, u);
        st3(pos2 + P, add(xp, dvs(scl(u, dt), 2)));
        break;
      case kAdvRK4K2:  // :118-135
        st3(k2 + P, u);
        st3(pos2 + P, add(xp, dvs(scl(u, dt), 2)));
        break;
      case kAdvRK4Upd: {  // :167-178, k3 used twice and k4 never (:173)
        const d3 a = ld3(k1 + P), b = ld3(k2 + P);
        const d3 s = add(add(add(a, scl(b, 2)), scl(u, 2)), u);
        st3(x + P, i > ignore ? add(xp, dvs(scl(s, dt), 6)) : add(xp, scl(a, dt)));
        break;
      }
      case kAdvAB2: {  // src/advect.cpp:181-217
        if (has_vprev && i >= 1) {
          const d3 vp = ld3(vprev + P);
          st3(x + P, add(xp, dvs(scl(sub(scl(u, 3), vp), dt), 2)));
        } else {
          st3(x + P, add(xp, scl(u, dt)));
        }
        st3(vprev + P, u);
        break;
      }
      default:
        break;
    }
  }
}

__global__ void copy_rows_kernel(const double* src, double* dst, int num, int PR, int row_elems, int from, int to,
                                 int rows) {
  const long long per = (long long)rows * row_elems;
  const long long total = per * num;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int n = (int)(k / per);
    const long long r = k % per;
    dst[((long long)n * PR + to) * row_elems + r] = src[((long long)n * PR + from) * row_elems + r];
  }
}

__global__ void extrapolate_kernel(double* x, const double* a, const double* b, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) x[k] = 2.0 * a[k] - b[k];
}

__global__ void check_finite_kernel(const double* x, long long n, int* flag) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    if (!isfinite(x[k])) atomicOr(flag, 1);
}

inline int grid_for(long long n, int bs = 256) {
  long long g = (n + bs - 1) / bs;
  if (g < 1) g = 1;
  if (g > 65535) g = 65535;
  return (int)g;
}

}  // namespace

Error launch_kinematics(const uvlm_kinematics* d_kin, WingShape ws, const double* pos_init, double* pos, double t,
                        cudaStream_t st) {
  const long long total = (long long)ws.num * (ws.R + 1) * (ws.C + 1);
  kinematics_kernel<<<grid_for(total), 256, 0, st>>>(d_kin, ws, pos_init, pos, t);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_shed(WingShape ws, const double* wing_pos, const double* wing_gamma, WakeLayout wl, double* wake_pos,
                  double* wake_gamma, bool shed_gamma, cudaStream_t st) {
  shed_kernel<<<grid_for(ws.num * (ws.C + 1)), 256, 0, st>>>(ws, wing_pos, wing_gamma, wl, wake_pos, wake_gamma,
                                                             shed_gamma ? 1 : 0);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_panel_geometry(const uvlm_kinematics* d_kin, WingShape ws, const double* pos, const double* pos_init,
                            double t, double* cx, double* cy, double* cz, double* normal, double* area, double* uls,
                            cudaStream_t st) {
  panel_geometry_kernel<<<grid_for((long long)ws.num * ws.R * ws.C), 256, 0, st>>>(d_kin, ws, pos, pos_init, t, cx, cy,
                                                                                   cz, normal, area, uls);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_assemble(WingShape ws, const double* pos, const double* cx, const double* cy, const double* cz,
                      const double* normal, bool fp32, void* A, bool out_f32, cudaStream_t st) {
  const long long N = (long long)ws.num * ws.R * ws.C;
  const long long lanes = N * ws.num * (ws.C + 1);
  const long long warps = (lanes + kAsmPerWarp - 1) / kAsmPerWarp;
  const unsigned grid = (unsigned)((warps + kAsmBlock / 32 - 1) / (kAsmBlock / 32));
  if (fp32) {
    if (out_f32)
      assemble_kernel<float, float><<<grid, kAsmBlock, 0, st>>>(ws, pos, cx, cy, cz, normal, (float*)A);
    else
      assemble_kernel<float, double><<<grid, kAsmBlock, 0, st>>>(ws, pos, cx, cy, cz, normal, (double*)A);
  } else {
    if (out_f32)
      assemble_kernel<double, float><<<grid, kAsmBlock, 0, st>>>(ws, pos, cx, cy, cz, normal, (float*)A);
    else
      assemble_kernel<double, double><<<grid, kAsmBlock, 0, st>>>(ws, pos, cx, cy, cz, normal, (double*)A);
  }
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_assemble_rings(const double* rings, int n, double* A, double* centroid, double* normal,
                            cudaStream_t st) {
  ring_geometry_kernel<<<grid_for(n), 256, 0, st>>>(rings, n, centroid, normal);
  UVLM_LAUNCH_CHECK();
  assemble_rings_kernel<<<grid_for((long long)n * n), 256, 0, st>>>(rings, n, centroid, normal, A);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_legacy_rhs(const uvlm_kinematics* d_kin, const int* d_kin_of, const double* rings0, int n,
                        const double* centroid, const double* normal, const double fs[3], double t,
                        const double* wake_vel, double* b, cudaStream_t st) {
  (void)centroid;
  legacy_rhs_kernel<<<grid_for(n), 256, 0, st>>>(d_kin, d_kin_of, rings0, n, normal, mk(fs[0], fs[1], fs[2]), t,
                                                 wake_vel, b);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_rhs(int N, const double* uw_x, const double* uw_y, const double* uw_z, const double* uls,
                 const double* normal, const double ff[3], double* b, cudaStream_t st) {
  rhs_kernel<<<grid_for(N), 256, 0, st>>>(N, uw_x, uw_y, uw_z, uls, normal, mk(ff[0], ff[1], ff[2]), b);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_line_prep(const uvlm_kinematics* d_kin, WingShape ws, const double* pos, const double* pos_init,
                       double t, double* tx, double* ty, double* tz, double* line_uls, cudaStream_t st) {
  line_prep_kernel<<<grid_for((long long)ws.num * ws.lines_per_wing()), 256, 0, st>>>(d_kin, ws, pos, pos_init, t, tx,
                                                                                      ty, tz, line_uls);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_loads(WingShape ws, const double* pos, const double* gamma, const double* gamma_prev,
                   const double* normal, const double* area, const double* vx, const double* vy, const double* vz,
                   const double* line_uls, const double ff[3], const double* chord_span, double t, double dt,
                   double* row, cudaStream_t st) {
  loads_kernel<512><<<ws.num, 512, 0, st>>>(ws, pos, gamma, gamma_prev, normal, area, vx, vy, vz, line_uls,
                                            mk(ff[0], ff[1], ff[2]), chord_span, t, dt, row);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_gather_wake(WakeLayout wl, const double* pos, double* tx, double* ty, double* tz, cudaStream_t st,
                         int first_row) {
  if (first_row < 1 || wl.node_rows <= first_row) return ok();
  gather_wake_kernel<<<grid_for((long long)wl.num * (wl.node_rows - first_row) * (wl.C + 1)), 256, 0, st>>>(
      wl, pos, first_row, tx, ty, tz);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_advect(AdvectMode mode, WakeLayout wl, double* x, double* pos2, double* k1, double* k2, double* k3,
                    double* vprev, bool has_vprev, const double* vx, const double* vy, const double* vz,
                    const double ff[3], double dt, int ignore_rows, cudaStream_t st, int vrow0) {
  if (wl.node_rows < 1) return ok();
  advect_kernel<<<grid_for((long long)wl.num * wl.node_rows * (wl.C + 1)), 256, 0, st>>>(
      (int)mode, wl, x, pos2, k1, k2, k3, vprev, has_vprev ? 1 : 0, vx, vy, vz, mk(ff[0], ff[1], ff[2]), dt,
      ignore_rows, vrow0);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_move_rows(double* buf, int num, int PR, int row_elems, int from, int to, int rows, double* tmp,
                       cudaStream_t st) {
  if (rows <= 0 || from == to) return ok();
  const long long total = (long long)num * rows * row_elems;
  copy_rows_kernel<<<grid_for(total), 256, 0, st>>>(buf, tmp, num, PR, row_elems, from, 0, rows);
  UVLM_LAUNCH_CHECK();
  copy_rows_kernel<<<grid_for(total), 256, 0, st>>>(tmp, buf, num, PR, row_elems, 0, to, rows);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_extrapolate(double* x, const double* a, const double* b, int n, cudaStream_t st) {
  extrapolate_kernel<<<grid_for(n), 256, 0, st>>>(x, a, b, n);
  UVLM_LAUNCH_CHECK();
  return ok();
}

Error launch_check_finite(const double* x, long long n, int* flag, cudaStream_t st) {
  check_finite_kernel<<<grid_for(n), 256, 0, st>>>(x, n, flag);
  UVLM_LAUNCH_CHECK();
  return ok();
}

}  // namespace uvlm
