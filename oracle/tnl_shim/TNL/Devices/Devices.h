// Minimal stand-in for the TNL device tags, written for this project so that the
// reference's header-only solver compiles with g++ on the host.  Both tags run on the
// host CPU: code that the reference launches on TNL::Devices::Cuda runs here through
// OpenMP, which is "the reference compiled for TNL::Devices::Host".
//
// This shim is test infrastructure (it only builds the oracle); it is never part of the
// product library.
#pragma once

#ifndef __cuda_callable__
#define __cuda_callable__
#endif
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif

namespace TNL {
namespace Devices {
struct Host {};
struct Cuda {};
}  // namespace Devices
}  // namespace TNL
