// bs_math.cuh -- Biot-Savart segment arithmetic shared by the N-body and the
// influence-matrix assembly (src/vortex.cpp:21-39).
#pragma once

#include "common.cuh"

namespace uvlm {
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

template <class T>
struct Node {
  T rx, ry, rz;  // x - p (zeroed when |x - p| < 1e-10)
  T ux, uy, uz;  // (x - p)/|x - p|
};

template <class T>
__device__ __forceinline__ Node<T> make_node(T x, T y, T z) {
  Node<T> nd;
  const T r2 = x * x + y * y + z * z;
  const bool ok = r2 >= (T)kCutR2;
  T inv;
  if constexpr (sizeof(T) == 4) {
    inv = ok ? rsqrt_approx(r2) : 0.f;
  } else {
    inv = ok ? rsqrt(r2) : 0.0;
  }
  nd.rx = ok ? x : (T)0;
  nd.ry = ok ? y : (T)0;
  nd.rz = ok ? z : (T)0;
  nd.ux = nd.rx * inv;
  nd.uy = nd.ry * inv;
  nd.uz = nd.rz * inv;
  return nd;
}

// Segment start=A -> end=B evaluated at x: r1 = x - A, r2 = x - B,
// d = r1 x r2, r0 = B - A = r1 - r2, K = g r0.(r1/|r1| - r2/|r2|) / |d|^2
// (src/vortex.cpp:24-38; g already carries 1/(4 pi)).
template <class T>
__device__ __forceinline__ void segment(const Node<T>& a, const Node<T>& b, T g, T& vx, T& vy, T& vz) {
  const T dx = a.ry * b.rz - a.rz * b.ry;
  const T dy = a.rz * b.rx - a.rx * b.rz;
  const T dz = a.rx * b.ry - a.ry * b.rx;
  const T d2 = dx * dx + dy * dy + dz * dz;
  const T dot = (a.rx - b.rx) * (a.ux - b.ux) + (a.ry - b.ry) * (a.uy - b.uy) + (a.rz - b.rz) * (a.uz - b.uz);
  T k;
  if constexpr (sizeof(T) == 4) {
    k = g * dot * rcp_approx(d2);
  } else {
    k = g * dot * __drcp_rn(d2);
  }
  k = (d2 < (T)kCutD2) ? (T)0 : k;
  vx += k * dx;
  vy += k * dy;
  vz += k * dz;
}

}  // namespace uvlm
