// step_math.cuh -- device arithmetic shared by the single-problem and the
// batched time-steppers: the Morphing kinematics and the load-line topology.
#pragma once

#include "../../include/uvlm_b200.h"
#include "common.cuh"
#include "step.cuh"

namespace uvlm {

// ------------------------------------------------------------ kinematics
// Morphing::Perfome (src/morphing.cpp:23-43) with PrepareMatrix (:54-76):
// x = plug(t) z + (attack * flap * twist) (x_ref + bend z), y<0 mirrored.
__device__ inline d3 perfome(const uvlm_kinematics& k, d3 x0, double t) {
  const d3 o = mk(k.origin[0], k.origin[1], k.origin[2]);
  d3 xr = sub(x0, o);
  const bool neg = xr.y < 0;
  if (neg) xr.y *= -1;
  const double phi = k.flap_amp * sin(k.flap_omega * t + k.flap_phase);
  const double alpha = k.alpha;
  const double beta = (k.twist_amp + k.twist_span_slope * fabs(xr.y)) * sin(k.twist_omega * t + k.twist_phase);
  const double F[3][3] = {{1, 0, 0}, {0, cos(phi), -sin(phi)}, {0, sin(phi), cos(phi)}};
  const double A[3][3] = {{cos(alpha), 0, sin(alpha)}, {0, 1, 0}, {-sin(alpha), 0, cos(alpha)}};
  const double T[3][3] = {{cos(beta), 0, sin(beta)}, {0, 1, 0}, {-sin(beta), 0, cos(beta)}};
  double AF[3][3], M[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) AF[i][j] = A[i][0] * F[0][j] + A[i][1] * F[1][j] + A[i][2] * F[2][j];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) M[i][j] = AF[i][0] * T[0][j] + AF[i][1] * T[1][j] + AF[i][2] * T[2][j];
  const double gz = k.plug_amp * sin(k.plug_omega * t + k.plug_phase);
  const double gb = (k.bend_cx * xr.x * (1 - xr.x) + k.bend_cy * xr.y * xr.y) * sin(k.bend_omega * t + k.bend_phase);
  const d3 v = mk(xr.x, xr.y, xr.z + gb);
  d3 x = mk(M[0][0] * v.x + M[0][1] * v.y + M[0][2] * v.z, M[1][0] * v.x + M[1][1] * v.y + M[1][2] * v.z,
            M[2][0] * v.x + M[2][1] * v.y + M[2][2] * v.z);
  x = add(mk(0, 0, gz), x);
  if (xr.y == 0) x.y = 0;
  if (neg) x.y *= -1;
  return add(x, o);
}

// Morphing::Velocity (src/morphing.cpp:45-52): central difference, h = 1e-6.
__device__ inline d3 morph_velocity(const uvlm_kinematics& k, d3 x0, double t) {
  const double h = 1e-6;
  const d3 x1 = perfome(k, x0, t - h);
  const d3 x2 = perfome(k, x0, t + h);
  return dvs(sub(x2, x1), 2 * h);
}

// Unique load lines of wing n: q < R*C spanwise S(i,j) (i < R, the TE row is
// skipped, joukowski.cpp:26), then R*(C+1) chordwise H(i,j).
__device__ inline void line_nodes(const WingShape& ws, int n, int q, long long& a, long long& b) {
  if (q < ws.R * ws.C) {
    const int i = q / ws.C, j = q % ws.C;
    a = ws.node(n, i, j);
    b = ws.node(n, i, j + 1);
  } else {
    q -= ws.R * ws.C;
    const int i = q / (ws.C + 1), j = q % (ws.C + 1);
    a = ws.node(n, i, j);
    b = ws.node(n, i + 1, j);
  }
}

__device__ inline double gam(const WingShape& ws, const double* g, int n, int i, int j) {
  if (i < 0 || i >= ws.R || j < 0 || j >= ws.C) return 0.0;
  return g[ws.ring(n, i, j)];
}

__device__ inline double line_strength(const WingShape& ws, const double* g, int n, int q) {
  if (q < ws.R * ws.C) {
    const int i = q / ws.C, j = q % ws.C;
    return gam(ws, g, n, i, j) - gam(ws, g, n, i - 1, j);
  }
  q -= ws.R * ws.C;
  const int i = q / (ws.C + 1), j = q % (ws.C + 1);
  return gam(ws, g, n, i, j - 1) - gam(ws, g, n, i, j);
}

}  // namespace uvlm
