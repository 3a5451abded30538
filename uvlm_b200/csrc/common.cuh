// common.cuh -- shared device/host helpers of the UVLM B200 library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

namespace uvlm {

constexpr double kPi = 3.14159265358979323846;
// Biot-Savart cut-off of src/vortex.cpp:31-35: |d|^2 < 1e-10 or |r| < 1e-10.
constexpr double kCutD2 = 1e-10;
constexpr double kCutR2 = 1e-20;  // |r| < 1e-10  <=>  |r|^2 < 1e-20

// Status codes of the C-ABI (mirrored in include/uvlm_b200.h).
enum Status : int {
  kOk = 0,
  kErrInvalid = 1,
  kErrCuda = 2,
  kErrSingular = 3,
  kErrNonFinite = 4,
  kErrState = 5,
  kErrCapacity = 6,
  kErrTimeout = 7,
  kErrUnsupported = 8,
};

struct Error {
  int code = kOk;
  std::string msg;
};

#define UVLM_CUDA_TRY(expr)                                                   \
  do {                                                                        \
    cudaError_t _e = (expr);                                                  \
    if (_e != cudaSuccess) {                                                  \
      return ::uvlm::Error{::uvlm::kErrCuda,                                   \
                           std::string(#expr ": ") + cudaGetErrorString(_e)}; \
    }                                                                         \
  } while (0)

// Every kernel launch of the library is followed by this check, which also
// counts the launch (uvlm_kernel_launch_count).
#define UVLM_LAUNCH_CHECK()          \
  do {                               \
    ::uvlm::note_launch();           \
    UVLM_CUDA_TRY(cudaGetLastError()); \
  } while (0)

#define UVLM_TRY(expr)                 \
  do {                                 \
    ::uvlm::Error _r = (expr);         \
    if (_r.code != ::uvlm::kOk) return _r; \
  } while (0)

inline Error ok() { return Error{}; }
// Process-wide count of kernel launches issued by the library (capi.cu).
void note_launch(int n = 1);
// FP32 FMA issue-rate probe (probe.cu).
Error measure_fp32_fma_peak(int num_sms, double* tflops);
Error measure_fp64_fma_peak(int num_sms, double* tflops);
// Message of the last failure of a context-free C-ABI call (capi.cu).
void set_global_error(const std::string& msg);
inline Error fail(int code, const std::string& m) { return Error{code, m}; }

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// --------------------------------------------------------- device helpers
struct d3 {
  double x, y, z;
};

__host__ __device__ inline d3 mk(double x, double y, double z) { return d3{x, y, z}; }
__host__ __device__ inline d3 add(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline d3 sub(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline d3 scl(d3 a, double s) { return d3{a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline d3 dvs(d3 a, double s) { return d3{a.x / s, a.y / s, a.z / s}; }
__host__ __device__ inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline d3 cross(d3 a, d3 b) {
  return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ inline double norm(d3 a) { return sqrt(dot(a, a)); }
__host__ __device__ inline d3 normalized(d3 a) {
  const double n = norm(a);
  return n > 0 ? dvs(a, n) : a;
}
__device__ inline d3 ld3(const double* p) { return d3{p[0], p[1], p[2]}; }
__device__ inline void st3(double* p, d3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

// Bounded waits: every spin loop and mbarrier wait of the library gives up
// after g_wait_limit clock cycles (default ~1 s at 2 GHz), sets an error word
// that the host turns into UVLM_ERR_TIMEOUT, and leaves the kernel.  The
// library is built without relocatable device code, so each translation unit
// holds its own copy of the limit; uvlm_set_wait_limit updates all of them
// through the per-unit setters below.
constexpr long long kDefaultWaitCycles = 2000000000LL;
static __device__ long long g_wait_limit = kDefaultWaitCycles;
// This translation unit's copy of the limit, on the current device.
static inline Error set_wait_limit_here(long long cycles) {
  const long long v = cycles > 0 ? cycles : kDefaultWaitCycles;
  UVLM_CUDA_TRY(cudaMemcpyToSymbol(g_wait_limit, &v, sizeof(v)));
  return ok();
}

}  // namespace uvlm
