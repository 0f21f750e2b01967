// Minimal TNL::Timer stand-in (wall clock).  Oracle-only test infrastructure.
#pragma once
#include <chrono>

namespace TNL {
class Timer {
 public:
  void reset() { elapsed_ = 0.0; running_ = false; }
  void start() { t0_ = std::chrono::steady_clock::now(); running_ = true; }
  void stop() {
    if (running_) elapsed_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    running_ = false;
  }
  double getRealTime() const { return elapsed_; }

 private:
  std::chrono::steady_clock::time_point t0_{};
  double elapsed_ = 0.0;
  bool running_ = false;
};
}  // namespace TNL
