#pragma once
// Query result types of the SdfOracle API (plugins/SdfOracle/include/
// SdfOracle/SdfCommon.h:10-37): the primary answer (signed gap, unit gap
// normal, witness point, valid flag) plus the per-feature candidates that
// contact-aware grids return (a single candidate otherwise).

#include <Eigen/Dense>
#include <array>
#include <vector>

namespace sdf {

inline constexpr int kMaxSdfQueryCandidates = 8;

struct SdfQueryCandidate
{
    double gap{0.0};
    Eigen::Vector3d gapNormal{1.0, 0.0, 0.0};
    Eigen::Vector3d witnessPoint{0.0, 0.0, 0.0};
    int branchId{-1};
};

struct SdfQueryResult
{
    double gap{0.0};
    Eigen::Vector3d gapNormal{1.0, 0.0, 0.0};
    Eigen::Vector3d witnessPoint{0.0, 0.0, 0.0};
    bool valid{false};
    std::vector<SdfQueryCandidate> candidates;
};

struct SdfFastQueryResult
{
    double gap{0.0};
    Eigen::Vector3d gapNormal{1.0, 0.0, 0.0};
    Eigen::Vector3d witnessPoint{0.0, 0.0, 0.0};
    bool valid{false};
    int candidateCount{0};
    std::array<SdfQueryCandidate, kMaxSdfQueryCandidates> candidates{};
};

} // namespace sdf
