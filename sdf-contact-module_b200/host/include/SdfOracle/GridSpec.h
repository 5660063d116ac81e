#pragma once
// Cell-centred voxel grid description shared by the builder, the queries and
// the SDFO file format.  Same fields and conventions as the SdfOracle plugin's
// GridSpec (plugins/SdfOracle/include/SdfOracle/GridSpec.h:17-74):
//   voxel centre  = bmin + voxel * (ijk + 0.5)
//   nearest voxel = round((p - bmin) / voxel - 0.5)
//   linear index  = i + nx * (j + ny * k)

#include <Eigen/Dense>
#include <algorithm>
#include <array>
#include <cmath>

namespace sdf {

struct GridSpec
{
    Eigen::Vector3d bmin{0.0, 0.0, 0.0};
    Eigen::Vector3d bmax{1.0, 1.0, 1.0};
    Eigen::Vector3d voxel{1.0, 1.0, 1.0};
    std::array<int, 3> shape{1, 1, 1};

    int nx() const { return shape[0]; }
    int ny() const { return shape[1]; }
    int nz() const { return shape[2]; }
    int totalVoxels() const { return shape[0] * shape[1] * shape[2]; }

    Eigen::Vector3d centerFromIndex(int i, int j, int k) const
    {
        return bmin + voxel.cwiseProduct(Eigen::Vector3d(i + 0.5, j + 0.5, k + 0.5));
    }

    void indexFromWorld(const Eigen::Vector3d& p, int& i, int& j, int& k) const
    {
        const Eigen::Vector3d f =
            (p - bmin).cwiseQuotient(voxel) - Eigen::Vector3d(0.5, 0.5, 0.5);
        i = static_cast<int>(std::round(f.x()));
        j = static_cast<int>(std::round(f.y()));
        k = static_cast<int>(std::round(f.z()));
    }

    bool inBounds(int i, int j, int k) const
    {
        return i >= 0 && j >= 0 && k >= 0 && i < shape[0] && j < shape[1] && k < shape[2];
    }

    int linearIndex(int i, int j, int k) const { return i + shape[0] * (j + shape[1] * k); }
};

// Smallest of {8, 16, ..., 2048} that is >= n, capped at maxRes (maxRes when
// n exceeds the ladder).
inline int snapToStandardResolution(int n, int maxRes)
{
    for (int v = 8; v <= 2048; v *= 2)
        if (v >= n || v >= maxRes) return std::min(v, maxRes);
    return maxRes;
}

} // namespace sdf
