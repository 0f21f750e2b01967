// Minimal TNL::Algorithms::reduce stand-in.  Runs sequentially in index order so the
// oracle's reductions are reproducible run to run (the reference's GPU reduction order
// is unspecified anyway).  Oracle-only test infrastructure.
#pragma once
#include <TNL/Devices/Devices.h>

namespace TNL {
namespace Algorithms {

template <typename Device, typename Index, typename Fetch, typename Reduction, typename Result>
Result reduce(Index begin, Index end, Fetch fetch, Reduction reduction, const Result& identity) {
  Result acc = identity;
  for (Index i = begin; i < end; ++i) acc = reduction(acc, fetch(i));
  return acc;
}

}  // namespace Algorithms
}  // namespace TNL
