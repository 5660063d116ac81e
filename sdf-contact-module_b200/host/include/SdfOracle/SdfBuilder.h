#pragma once
// SDF grid construction (plugins/SdfOracle/include/SdfOracle/SdfBuilder.h:
// 24-113), executed on the GPU through libsdfo_cuda: the signed distance,
// normal, witness point and Hessian of every voxel (dense) or of every voxel
// of the narrow-band blocks (sparse).  Same parameters and defaults; results
// are identical to the reference's CPU builder.

#include <functional>
#include <string>

#include "SdfOracle/SdfData.h"
#include "SdfOracle/SdfSurfaceMesh.h"

namespace sdf {

struct BuilderParams
{
    double padding{0.1};       ///< padding as a fraction of the bounding-box diagonal
    double voxelSize{0.0};     ///< explicit voxel size (0 = longest side / targetResolution)
    int targetResolution{128}; ///< voxels along the longest padded side
    int maxResolution{512};    ///< cap on voxels along any axis
    std::function<void(const std::string&)> logCallback; ///< optional progress logger
};

struct SparseBuilderParams : public BuilderParams
{
    int blockDim{8};
    int haloVoxels{2};
    int bandVoxels{8};
    double bandDistance{0.0}; ///< explicit narrow-band half width (0 = bandVoxels * voxel)
    bool storeHessian{true};
};

struct ContactAwareBuilderParams : public BuilderParams
{
    int maxCandidates{4};
    double featureDistanceTolerance{0.0};
    double normalMergeAngleDegrees{5.0};
    int tileDim{8};
    bool useTileAcceleration{true};
    bool storeHessian{true};
    bool sparse{false};
    int blockDim{8};
    int haloVoxels{2};
    int bandVoxels{8};
    double bandDistance{0.0};
};

class SdfBuilder
{
public:
    static SdfData build(const std::vector<Eigen::Vector3d>& vertices,
                         const std::vector<std::array<int, 3>>& triangles,
                         const BuilderParams& params = {});
    static SdfData build(const TriangleMesh& mesh, const BuilderParams& params = {});

    /// Contact-aware builds are not provided by the GPU backend yet: these
    /// throw std::runtime_error.
    static SdfData buildContactAware(const CornerNormalTriangleMesh& mesh,
                                     const ContactAwareBuilderParams& params = {});
    static SparseSdfData buildSparseContactAware(const CornerNormalTriangleMesh& mesh,
                                                 const ContactAwareBuilderParams& params = {});

    static SparseSdfData buildSparse(const std::vector<Eigen::Vector3d>& vertices,
                                     const std::vector<std::array<int, 3>>& triangles,
                                     const SparseBuilderParams& params = {});
    static SparseSdfData buildSparse(const TriangleMesh& mesh,
                                     const SparseBuilderParams& params = {});
};

} // namespace sdf
