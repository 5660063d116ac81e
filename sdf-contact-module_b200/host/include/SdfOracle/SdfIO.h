#pragma once
// The "SDFO" v0.1.0 binary grid file (plugins/SdfOracle/include/SdfOracle/
// SdfIO.h:1-45; layout in plugins/SdfOracle/src/SdfIO.cpp:60-552): a 128-byte
// header (magic, version 100, shape, bmin, bmax, voxel, flags, layout fields)
// followed by the dense FP64 or sparse FP32 block payload.  Byte-compatible
// with the reference in both directions.

#include <string>

#include "SdfOracle/SdfData.h"

namespace sdf {

bool saveSdf(const SdfData& data, const std::string& path);
SdfData loadSdf(const std::string& path);
bool saveSparseSdf(const SparseSdfData& data, const std::string& path);
SparseSdfData loadSparseSdf(const std::string& path);
bool isValidSdf(const std::string& path);
bool isSparseSdf(const std::string& path);

} // namespace sdf
