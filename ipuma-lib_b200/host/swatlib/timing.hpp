// Wall-clock timer with tick/tock accumulation (src/swatlib/timing.hpp:27-65).
#ifndef IPUMA_B200_SWATLIB_TIMING_HPP
#define IPUMA_B200_SWATLIB_TIMING_HPP
#include <chrono>

namespace swatlib {
class TickTock {
  using clock = std::chrono::steady_clock;
  clock::time_point t1, t2;
  long long accumulated_us = 0;

 public:
  void tick() { t1 = clock::now(); }
  void tock() {
    t2 = clock::now();
    accumulated_us += std::chrono::duration_cast<std::chrono::microseconds>(t2 - t1).count();
  }
  template <typename D = std::chrono::milliseconds>
  long long duration() const {
    return std::chrono::duration_cast<D>(t2 - t1).count();
  }
  long long accumulate_microseconds() const { return accumulated_us; }
};
}  // namespace swatlib
#endif
