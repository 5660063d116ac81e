#pragma once
// Integration alias kept from the plugin (plugins/SdfOracle/include/
// SdfOracle/NexDynAdapter.h:17): hosts that name the standalone oracle keep
// compiling against the GPU-backed one.

#include "SdfOracle/SdfOracle.h"

namespace sdf {

using StandaloneSdfOracle = SdfOracle;

} // namespace sdf
