// fatal_mode.cpp -- the C++ adapter's error behaviour, without a GPU: a
// failing call throws UVLM::Error by default; built with
// -DUVLM_B200_FATAL_ON_ERROR it prints the message and aborts, as the
// reference's LOG(FATAL) / CHECK does.  The failing call is a host-only one
// (a state record with no path).
#include <cstdio>

#include "uvlm_b200.hpp"

int main() {
  try {
    UVLM::detail::check(uvlm_write_state_record(nullptr, 0, UVLM_OUTPUT_SHEETS, 0, 0, 0, 0, nullptr, nullptr, nullptr,
                                                nullptr, 0.0),
                        "WriteStateRecord");
  } catch (const UVLM::Error& e) {
    std::printf("caught %d: %s\n", e.code(), e.what());
    return 0;
  }
  return 1;
}
