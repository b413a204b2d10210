// Stand-in for Kokkos_Timer.hpp (included but unused by the reference).
#pragma once
#include <chrono>

namespace Kokkos {
class Timer {
  std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();

 public:
  void reset() { t0_ = std::chrono::steady_clock::now(); }
  double seconds() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }
};
}  // namespace Kokkos
