// noalloc.cu -- InducedVelocity over a vortex-ring sheet set without any
// device allocation.
//
// Some callers cannot call cudaMalloc: real-time loops in which cudaMalloc or
// cudaFree would synchronise the whole device, and host frameworks that budget
// all device memory themselves and hand out only buffers they own.  This entry
// point computes the same velocities as uvlm_sheet_induced_velocity, but its
// inputs and outputs are device pointers owned by the caller and all of its
// scratch (the source records, the per-split partial sums and the SoA
// target/velocity vectors) lives in one file-scope device array of
// kNoAllocScratchBytes (32 MiB).  Every GPU that loads this library holds that
// array until the process exits.
//
// The array is shared by every call and keeps the previous call's contents;
// nothing in it needs to start at zero (every byte a call reads was written by
// the same call, and the empty-sheet case clears the velocities it returns).
// Calls that overlap on the GPU (for example on two streams) race on the
// array: serialise them.
#include <cuda.h>

#include <climits>
#include <mutex>

#include "../../include/uvlm_b200.h"
#include "device_once.h"
#include "nbody.cuh"

namespace uvlm {
namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;

// Device-side scratch.  In host code this name is only a stand-in: its device
// address comes from cudaGetSymbolAddress (scratch_address below).
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // context the address belongs to

// Unique id of the context current on this thread (0 if the driver entry
// points are unavailable).  A cudaDeviceReset destroys the primary context and
// the module with it; the next primary context has another id, so the address
// is looked up again instead of reusing a stale one.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(fn);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(fn);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx) get_id(ctx, &id);
  return id;
}

// Set-up, once per device (and again only if that device's context was
// reset), with that device current: the device address of the scratch array.
// The first call on a device does this set-up, so that first call should come
// before any stream capture.
Error scratch_address(void** out) {
  int dev = 0;
  UVLM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(kErrUnsupported, "device ordinal out of range");
  UVLM_CUDA_TRY(cudaSetDevice(dev));  // makes the device's primary context current on this thread
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(kErrCuda, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return ok();
}

__global__ void noalloc_aos_to_soa(const double* a, long long n, double* x, double* y, double* z) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    x[k] = a[3 * k];
    y[k] = a[3 * k + 1];
    z[k] = a[3 * k + 2];
  }
}

__global__ void noalloc_soa_to_aos(const double* x, const double* y, const double* z, long long n, double* a) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    a[3 * k] = x[k];
    a[3 * k + 1] = y[k];
    a[3 * k + 2] = z[k];
  }
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
inline int grid1d(long long n) { return (int)std::min<long long>(std::max<long long>((n + 255) / 256, 1), 4096); }

Error run_noalloc(const double* pos, const double* gamma, int64_t num, int64_t grows, int64_t gcols,
                  const double* targets, int64_t n_targets, double* out, int32_t precision, cudaStream_t st) {
  if (!targets || !out || num < 0 || grows < 0 || gcols < 0 || n_targets < 0)
    return fail(kErrInvalid, "invalid argument");
  // the sheet shape is held in int fields of the N-body views
  if (num > INT_MAX || grows >= INT_MAX || gcols >= INT_MAX) return fail(kErrCapacity, "sheet shape too large");
  // pos and gamma are read only when the sheet set has rings
  const bool has_rings = num > 0 && grows > 0 && gcols > 0;
  if (has_rings && (!pos || !gamma)) return fail(kErrInvalid, "invalid argument");
  if (n_targets == 0) return ok();
  const NBodyPrec prec = precision == UVLM_PRECISION_MIXED ? kNBodyFP32 : kNBodyFP64;
  const size_t rec_size = prec == kNBodyFP32 ? sizeof(RecF) : sizeof(RecD);
  // bound every factor by division before multiplying, so that no product
  // can wrap around before the capacity check
  const unsigned long long cap = kNoAllocScratchBytes;
  const unsigned long long max_nodes = cap / rec_size;
  const unsigned long long nr = (unsigned long long)grows + 1, nc = (unsigned long long)gcols + 1;
  if (has_rings && ((unsigned long long)num > max_nodes || nr > max_nodes / (unsigned long long)num ||
                    nc > max_nodes / ((unsigned long long)num * nr)))
    return fail(kErrCapacity, "the sheet needs more than the allocation-free entry point's " + std::to_string(cap) +
                                  " bytes of scratch");
  if ((unsigned long long)n_targets > cap / (9 * sizeof(double)))
    return fail(kErrCapacity, "the target set needs more than the allocation-free entry point's " +
                                  std::to_string(cap) + " bytes of scratch");
  const long long nodes = has_rings ? (long long)((unsigned long long)num * nr * nc) : 0;
  const size_t rec_bytes = align256((size_t)nodes * rec_size);
  const size_t vec_bytes = align256(sizeof(double) * (size_t)n_targets);
  const size_t fixed = rec_bytes + 6 * vec_bytes;
  const size_t one_split = sizeof(double) * 3 * (size_t)n_targets;
  if (fixed + one_split > kNoAllocScratchBytes)
    return fail(kErrCapacity, "sheet and target set need " + std::to_string(fixed + one_split) +
                                  " bytes of scratch; the allocation-free entry point has " +
                                  std::to_string(kNoAllocScratchBytes));
  void* base = nullptr;
  UVLM_TRY(scratch_address(&base));
  unsigned char* p = static_cast<unsigned char*>(base);
  double* tx = reinterpret_cast<double*>(p);
  double* ty = reinterpret_cast<double*>(p + vec_bytes);
  double* tz = reinterpret_cast<double*>(p + 2 * vec_bytes);
  double* vx = reinterpret_cast<double*>(p + 3 * vec_bytes);
  double* vy = reinterpret_cast<double*>(p + 4 * vec_bytes);
  double* vz = reinterpret_cast<double*>(p + 5 * vec_bytes);
  NBodyWork w;
  w.records = p + 6 * vec_bytes;
  w.records_cap = (long long)rec_bytes;
  w.partial = reinterpret_cast<double*>(p + fixed);
  w.partial_cap = (long long)((kNoAllocScratchBytes - fixed) / sizeof(double));
  w.max_splits = (long long)((kNoAllocScratchBytes - fixed) / one_split);
  noalloc_aos_to_soa<<<grid1d(n_targets), 256, 0, st>>>(targets, n_targets, tx, ty, tz);
  UVLM_LAUNCH_CHECK();
  if (has_rings) {
    SheetView v{pos, (int)grows + 1, 0, gamma, (int)grows, 0, (int)num, (int)grows + 1, (int)gcols};
    SourceBlock blk;
    UVLM_TRY(nbody_build_sources(&v, 1, prec, &w, &blk, st));
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    UVLM_TRY(nbody_eval(&blk, 1, prec, tx, ty, tz, n_targets, vx, vy, vz, &w, prec == kNBodyFP32 ? 16 : 9, sms, st));
  } else {
    UVLM_CUDA_TRY(cudaMemsetAsync(vx, 0, 3 * vec_bytes, st));
  }
  noalloc_soa_to_aos<<<grid1d(n_targets), 256, 0, st>>>(vx, vy, vz, n_targets, out);
  UVLM_LAUNCH_CHECK();
  return ok();
}

}  // namespace
}  // namespace uvlm

extern "C" int uvlm_sheet_induced_velocity_noalloc(const double* pos, const double* gamma, int64_t num,
                                                   int64_t grows, int64_t gcols, const double* targets,
                                                   int64_t n_targets, double* out, int32_t precision,
                                                   void* stream) {
  const uvlm::Error e = uvlm::run_noalloc(pos, gamma, num, grows, gcols, targets, n_targets, out, precision,
                                          static_cast<cudaStream_t>(stream));
  if (e.code) uvlm::set_global_error(e.msg);
  return e.code;
}
