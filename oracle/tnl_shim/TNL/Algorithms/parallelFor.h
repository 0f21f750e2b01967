// Minimal TNL::Algorithms::parallelFor stand-in: every device tag runs on the host with
// OpenMP.  1-D ranges pass the int index; 2-D and 3-D StaticArray ranges pass the
// multi-index with the first component fastest (the order TNL documents).  The
// reference's in-place periodic-shift update touches every (direction, address) pair
// from exactly one cell, so the result does not depend on the thread schedule.
//
// Oracle-only test infrastructure.
#pragma once
#include <type_traits>

#include <TNL/Containers/StaticArray.h>
#include <TNL/Devices/Devices.h>

namespace TNL {
namespace Algorithms {

template <typename Device, typename IndexB, typename IndexE, typename Func,
          typename = std::enable_if_t<std::is_integral_v<IndexB> && std::is_integral_v<IndexE>>>
void parallelFor(IndexB begin, IndexE end, Func f) {
#pragma omp parallel for schedule(static) firstprivate(f)
  for (long long i = static_cast<long long>(begin); i < static_cast<long long>(end); ++i) {
    f(static_cast<int>(i));
  }
}

template <typename Device, typename T, typename Func>
void parallelFor(const Containers::StaticArray<2, T>& begin, const Containers::StaticArray<2, T>& end,
                 Func f) {
  const long long n0 = end[0] - begin[0];
  const long long n1 = end[1] - begin[1];
  if (n0 <= 0 || n1 <= 0) return;
#pragma omp parallel for schedule(static) firstprivate(f)
  for (long long t = 0; t < n0 * n1; ++t) {
    Containers::StaticArray<2, T> idx{static_cast<T>(begin[0] + t % n0), static_cast<T>(begin[1] + t / n0)};
    f(idx);
  }
}

template <typename Device, typename T, typename Func>
void parallelFor(const Containers::StaticArray<3, T>& begin, const Containers::StaticArray<3, T>& end,
                 Func f) {
  const long long n0 = end[0] - begin[0];
  const long long n1 = end[1] - begin[1];
  const long long n2 = end[2] - begin[2];
  if (n0 <= 0 || n1 <= 0 || n2 <= 0) return;
#pragma omp parallel for schedule(static) firstprivate(f)
  for (long long t = 0; t < n0 * n1 * n2; ++t) {
    Containers::StaticArray<3, T> idx{static_cast<T>(begin[0] + t % n0),
                                      static_cast<T>(begin[1] + (t / n0) % n1),
                                      static_cast<T>(begin[2] + t / (n0 * n1))};
    f(idx);
  }
}

}  // namespace Algorithms
}  // namespace TNL
