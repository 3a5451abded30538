// device_once.h -- per-device "do this once" guards for kernel attributes.
//
// cudaFuncSetAttribute (for example the dynamic shared-memory limit of a
// kernel that needs more than 48 KB) applies to the device that is current
// when it is called.  A process that drives several GPUs (one context per
// device, or the allocation-free entry point called on several ordinals) must
// therefore apply it once on EVERY device, not once per process.  This header
// holds the bookkeeping; it is plain C++ (no CUDA types) so that the logic is
// unit-tested on the host.
#pragma once

#include <atomic>

namespace uvlm {

constexpr int kMaxDevices = 64;

// Outcome of a per-device set-up: 0 not yet run, 1 succeeded, -1 failed.
struct PerDeviceOnce {
  std::atomic<int> state[kMaxDevices];
  PerDeviceOnce() {
    for (auto& s : state) s.store(0, std::memory_order_relaxed);
  }
};

// Runs fn() (returning true on success) the first time it is called for
// `device` and remembers the outcome; later calls for that device return the
// remembered outcome without running fn.  Concurrent first calls may both run
// fn, which is harmless for idempotent set-ups such as attribute setters.
// Ordinals outside [0, kMaxDevices) run fn every time.
template <class F>
bool once_on_device(PerDeviceOnce& once, int device, F&& fn) {
  if (device < 0 || device >= kMaxDevices) return fn();
  int s = once.state[device].load(std::memory_order_acquire);
  if (s == 0) {
    s = fn() ? 1 : -1;
    once.state[device].store(s, std::memory_order_release);
  }
  return s > 0;
}

}  // namespace uvlm
