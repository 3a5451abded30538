// refapi_util.cuh -- helpers shared by the context-free C-ABI entry points
// (refapi.cu, legacy.cu): scoped device scratch, AoS/SoA conversion, AoS
// rings as 1 x 1 sheets, the FP64/FP32 N-body at arbitrary targets and a
// fixed-order block sum.
#pragma once

#include <algorithm>
#include <vector>

#include "../../include/uvlm_b200.h"
#include "common.cuh"
#include "nbody.cuh"

using namespace uvlm;

namespace {

int report(const Error& e) {
  if (e.code) set_global_error(e.msg);
  return e.code;
}

int sms() {
  int d = 0, v = 148;
  cudaGetDevice(&d);
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
  return v;
}

// Device buffers freed at scope exit.
struct Scratch {
  std::vector<void*> p;
  ~Scratch() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  Error get(T** out, size_t count) {
    *out = nullptr;
    if (count == 0) return ok();
    UVLM_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(out), sizeof(T) * count));
    p.push_back(*out);
    return ok();
  }
  template <class T>
  Error up(T** out, const T* host, size_t count) {
    UVLM_TRY(get(out, count));
    if (count) UVLM_CUDA_TRY(cudaMemcpy(*out, host, sizeof(T) * count, cudaMemcpyHostToDevice));
    return ok();
  }
};

__global__ void aos_to_soa(const double* a, long long n, double* x, double* y, double* z) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    x[k] = a[3 * k];
    y[k] = a[3 * k + 1];
    z[k] = a[3 * k + 2];
  }
}
__global__ void soa_to_aos(const double* x, const double* y, const double* z, long long n, double* a, const double* add3,
                           const double* base, double scale) {
  // a = base + (v + add3) * scale   (base/add3 may be NULL)
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    double v[3] = {x[k], y[k], z[k]};
    for (int d = 0; d < 3; ++d) {
      double u = v[d] + (add3 ? add3[d] : 0.0);
      a[3 * k + d] = base ? base[3 * k + d] + u * scale : u;
    }
  }
}
// AoS ring k (nodes n0..n3) -> 1 x 1 sheet k with p(0,0)=n0, p(0,1)=n1,
// p(1,1)=n2, p(1,0)=n3 and circulation -g: the sheet walks n0->n1->n2->n3,
// the AoS ring nodes[k+1]->nodes[k] (src/vortex.h:132-140).
__global__ void rings_to_sheets(const double* rings, const double* g, long long n, double* pos, double* gam) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const double* r = rings + 12 * k;
    double* p = pos + 12 * k;
    const int map[4] = {0, 1, 3, 2};  // sheet order (0,0),(0,1),(1,0),(1,1)
    for (int q = 0; q < 4; ++q)
      for (int d = 0; d < 3; ++d) p[3 * q + d] = r[3 * map[q] + d];
    gam[k] = -g[k];
  }
}
constexpr int kSumThreads = 256;

__device__ inline d3 block_sum3(d3 v, double* sh) {
  for (int off = 16; off; off >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, off);
    v.y += __shfl_down_sync(0xffffffffu, v.y, off);
    v.z += __shfl_down_sync(0xffffffffu, v.z, off);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    sh[3 * wid] = v.x;
    sh[3 * wid + 1] = v.y;
    sh[3 * wid + 2] = v.z;
  }
  __syncthreads();
  d3 r = mk(0, 0, 0);
  for (int w = 0; w < kSumThreads / 32; ++w) r = add(r, mk(sh[3 * w], sh[3 * w + 1], sh[3 * w + 2]));
  return r;
}

inline int gfor(long long n) { return (int)std::min<long long>(std::max<long long>((n + 255) / 256, 1), 65535); }

Error velocity_at(const SheetView* views, int nv, NBodyPrec prec, const double* d_targets_aos, long long nt,
                  double* vx, double* vy, double* vz, Scratch& S) {
  double *tx, *ty, *tz;
  UVLM_TRY(S.get(&tx, nt));
  UVLM_TRY(S.get(&ty, nt));
  UVLM_TRY(S.get(&tz, nt));
  aos_to_soa<<<gfor(nt), 256>>>(d_targets_aos, nt, tx, ty, tz);
  UVLM_LAUNCH_CHECK();
  NBodyWork w;
  long long recs = 0;
  for (int i = 0; i < nv; ++i) recs += (long long)views[i].num * views[i].node_rows * (views[i].cols + 1);
  w.records_cap = std::max<long long>(recs, 1) * (long long)sizeof(RecD);
  UVLM_TRY(S.get(reinterpret_cast<char**>(&w.records), (size_t)w.records_cap));
  w.partial_cap = 3 * std::max<long long>(nt, 1) * 64;
  UVLM_TRY(S.get(&w.partial, (size_t)w.partial_cap));
  SourceBlock blocks[4];
  UVLM_TRY(nbody_build_sources(views, nv, prec, &w, blocks, 0));
  const int variant = prec == kNBodyFP32 ? 16 : 9;  // fp32_h3_t2_b128_x2f, fp64_h2_t1_b128_m3
  UVLM_TRY(nbody_eval(blocks, nv, prec, tx, ty, tz, nt, vx, vy, vz, &w, variant, sms(), 0));
  return ok();
}

}  // namespace
