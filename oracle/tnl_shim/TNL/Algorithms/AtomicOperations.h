// Placeholder for TNL::Algorithms::AtomicOperations: the reference includes it from
// types.h, but only its STL voxeliser (not on the lattice-update path) uses it.
// Oracle-only test infrastructure.
#pragma once
#include <TNL/Devices/Devices.h>
