// Host-side test of the per-device once-guard of kernel attributes
// (uvlm_b200/csrc/device_once.h): the set-up runs once on every device, its
// outcome is remembered per device, and concurrent first calls agree.
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

#include "device_once.h"

#define CHECK(c)                                                   \
  do {                                                             \
    if (!(c)) {                                                    \
      std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #c);   \
      return 1;                                                    \
    }                                                              \
  } while (0)

int main() {
  using uvlm::once_on_device;
  uvlm::PerDeviceOnce once;
  int runs[uvlm::kMaxDevices] = {};
  auto setup = [&](int dev) { return once_on_device(once, dev, [&] { runs[dev]++; return true; }); };
  // device 0 twice, device 1 once: two set-ups, not one per process
  CHECK(setup(0));
  CHECK(setup(0));
  CHECK(setup(1));
  CHECK(runs[0] == 1 && runs[1] == 1);
  // a failed set-up is remembered for its device only
  uvlm::PerDeviceOnce failing;
  int fails = 0;
  CHECK(!once_on_device(failing, 3, [&] { fails++; return false; }));
  CHECK(!once_on_device(failing, 3, [&] { fails++; return true; }));
  CHECK(fails == 1);
  CHECK(once_on_device(failing, 4, [&] { return true; }));
  // ordinals outside the table run the set-up every time
  int outside = 0;
  CHECK(once_on_device(once, uvlm::kMaxDevices, [&] { outside++; return true; }));
  CHECK(once_on_device(once, -1, [&] { outside++; return true; }));
  CHECK(outside == 2);
  // many threads on many devices: every call sees success, every device set up
  uvlm::PerDeviceOnce shared;
  std::atomic<int> per_dev[8];
  for (auto& a : per_dev) a = 0;
  std::atomic<int> bad{0};
  std::vector<std::thread> th;
  for (int t = 0; t < 16; ++t)
    th.emplace_back([&, t] {
      for (int k = 0; k < 1000; ++k) {
        const int d = (t + k) % 8;
        if (!once_on_device(shared, d, [&] { per_dev[d]++; return true; })) bad++;
      }
    });
  for (auto& x : th) x.join();
  CHECK(bad == 0);
  for (auto& a : per_dev) CHECK(a >= 1);
  std::printf("device_once ok\n");
  return 0;
}
