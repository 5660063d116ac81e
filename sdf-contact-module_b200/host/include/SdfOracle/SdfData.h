#pragma once
// Host-side grid containers of the SdfOracle API (plugins/SdfOracle/include/
// SdfOracle/SdfData.h:27-303), field for field:
//   SdfData        dense FP64: phi0, unit normal n0, symmetric Hessian H0 and
//                  closest surface point witness0 per voxel (x-fastest), plus
//                  optional contact-aware candidates
//   SparseSdfBlock one blockDim^3 block of FP32 phi / normal / Hessian
//   SparseSdfData  the stored blocks and a key -> block index map
// These are what SdfBuilder returns, what SdfOracle is constructed from and
// what the SDFO file holds; the GPU copy lives behind the oracle's handle.

#include <Eigen/Dense>
#include <algorithm>
#include <array>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "SdfOracle/GridSpec.h"
#include "SdfOracle/SdfCommon.h"

namespace sdf {

struct SdfData
{
    static constexpr int kMaxContactCandidates = kMaxSdfQueryCandidates;

    GridSpec spec;
    std::vector<double> phi0;
    std::vector<Eigen::Vector3d> n0;
    std::vector<Eigen::Matrix3d> H0;
    std::vector<Eigen::Vector3d> witness0;

    int contactCandidateStride{0};
    std::vector<uint8_t> contactCandidateCount;
    std::vector<double> contactCandidatePhi0;
    std::vector<Eigen::Vector3d> contactCandidateNormal0;
    std::vector<int32_t> contactCandidateBranchId;

    void resize(const GridSpec& s)
    {
        spec = s;
        const size_t n = static_cast<size_t>(s.totalVoxels());
        phi0.assign(n, 0.0);
        n0.assign(n, Eigen::Vector3d::UnitX());
        H0.assign(n, Eigen::Matrix3d::Zero());
        witness0.assign(n, Eigen::Vector3d::Zero());
        clearContactCandidates();
    }

    void resizeContactCandidates(int maxCandidates)
    {
        contactCandidateStride = std::max(0, std::min(maxCandidates, kMaxContactCandidates));
        const size_t n = static_cast<size_t>(spec.totalVoxels());
        const size_t m = n * static_cast<size_t>(contactCandidateStride);
        contactCandidateCount.assign(n, 0);
        contactCandidatePhi0.assign(m, 0.0);
        contactCandidateNormal0.assign(m, Eigen::Vector3d::UnitX());
        contactCandidateBranchId.assign(m, -1);
    }

    void clearContactCandidates()
    {
        contactCandidateStride = 0;
        contactCandidateCount.clear();
        contactCandidatePhi0.clear();
        contactCandidateNormal0.clear();
        contactCandidateBranchId.clear();
    }

    bool hasContactCandidates() const
    {
        const size_t n = static_cast<size_t>(spec.totalVoxels());
        const size_t m = n * static_cast<size_t>(contactCandidateStride);
        return contactCandidateStride > 0 && contactCandidateCount.size() == n &&
               contactCandidatePhi0.size() == m && contactCandidateNormal0.size() == m &&
               contactCandidateBranchId.size() == m;
    }

    int contactCandidateIndex(int voxelIndex, int candidateIndex) const
    {
        return voxelIndex * contactCandidateStride + candidateIndex;
    }

    double& phi(int i, int j, int k) { return phi0[spec.linearIndex(i, j, k)]; }
    double phi(int i, int j, int k) const { return phi0[spec.linearIndex(i, j, k)]; }
    Eigen::Vector3d& normal(int i, int j, int k) { return n0[spec.linearIndex(i, j, k)]; }
    const Eigen::Vector3d& normal(int i, int j, int k) const { return n0[spec.linearIndex(i, j, k)]; }
    Eigen::Matrix3d& hessian(int i, int j, int k) { return H0[spec.linearIndex(i, j, k)]; }
    const Eigen::Matrix3d& hessian(int i, int j, int k) const { return H0[spec.linearIndex(i, j, k)]; }
    Eigen::Vector3d& witness(int i, int j, int k) { return witness0[spec.linearIndex(i, j, k)]; }
    const Eigen::Vector3d& witness(int i, int j, int k) const { return witness0[spec.linearIndex(i, j, k)]; }
};

struct SparseSdfBlock
{
    std::array<int, 3> index{0, 0, 0};
    std::vector<float> phi0;
    std::vector<float> normal0;  // x, y, z per local voxel
    std::vector<float> hessian0; // xx, xy, xz, yy, yz, zz per local voxel
    std::vector<uint8_t> contactCandidateCount;
    std::vector<float> contactCandidatePhi0;
    std::vector<float> contactCandidateNormal0;
    std::vector<int32_t> contactCandidateBranchId;

    int localIndex(int x, int y, int z, int blockDim) const
    {
        return x + blockDim * (y + blockDim * z);
    }

    int contactCandidateIndex(int localVoxelIndex, int candidateIndex, int stride) const
    {
        return localVoxelIndex * stride + candidateIndex;
    }

    bool hasContactCandidates(int blockVoxelCount, int stride) const
    {
        const size_t v = static_cast<size_t>(blockVoxelCount), m = v * static_cast<size_t>(stride);
        return stride > 0 && contactCandidateCount.size() >= v && contactCandidatePhi0.size() >= m &&
               contactCandidateNormal0.size() >= 3 * m && contactCandidateBranchId.size() >= m;
    }
};

struct SparseSdfData
{
    GridSpec spec;
    int blockDim{8};
    int haloVoxels{2};
    double bandDistance{0.0};
    bool hasHessian{true};
    int contactCandidateStride{0};
    std::vector<SparseSdfBlock> blocks;
    std::unordered_map<uint64_t, size_t> blockLookup;

    // 21 bits per block coordinate, bi in the low bits.
    static uint64_t key(int bi, int bj, int bk)
    {
        return static_cast<uint64_t>(static_cast<uint32_t>(bi)) |
               (static_cast<uint64_t>(static_cast<uint32_t>(bj)) << 21) |
               (static_cast<uint64_t>(static_cast<uint32_t>(bk)) << 42);
    }

    void rebuildIndex()
    {
        blockLookup.clear();
        blockLookup.reserve(blocks.size());
        for (size_t b = 0; b < blocks.size(); ++b)
            blockLookup.emplace(key(blocks[b].index[0], blocks[b].index[1], blocks[b].index[2]), b);
    }

    bool empty() const { return blocks.empty(); }
    int blockVoxelCount() const { return blockDim * blockDim * blockDim; }
    size_t totalStoredVoxels() const { return blocks.size() * static_cast<size_t>(blockVoxelCount()); }

    bool hasContactCandidates() const
    {
        if (contactCandidateStride <= 0 || blocks.empty()) return false;
        for (const SparseSdfBlock& b : blocks)
            if (!b.hasContactCandidates(blockVoxelCount(), contactCandidateStride)) return false;
        return true;
    }

    const SparseSdfBlock* blockForVoxel(int i, int j, int k) const
    {
        if (!spec.inBounds(i, j, k) || blockDim <= 0) return nullptr;
        const auto it = blockLookup.find(key(i / blockDim, j / blockDim, k / blockDim));
        return it == blockLookup.end() ? nullptr : &blocks[it->second];
    }

    bool sample(int i, int j, int k, double& phi, Eigen::Vector3d& normal,
                Eigen::Matrix3d* hessian = nullptr) const
    {
        const SparseSdfBlock* b = blockForVoxel(i, j, k);
        return b != nullptr && sampleFromBlock(*b, i, j, k, phi, normal, hessian);
    }

    bool sampleFromBlock(const SparseSdfBlock& block, int i, int j, int k, double& phi,
                         Eigen::Vector3d& normal, Eigen::Matrix3d* hessian = nullptr) const
    {
        const int lx = i - block.index[0] * blockDim;
        const int ly = j - block.index[1] * blockDim;
        const int lz = k - block.index[2] * blockDim;
        if (lx < 0 || ly < 0 || lz < 0 || lx >= blockDim || ly >= blockDim || lz >= blockDim)
            return false;
        const int v = blockVoxelCount();
        const int local = block.localIndex(lx, ly, lz, blockDim);
        if (block.phi0.size() < static_cast<size_t>(v) ||
            block.normal0.size() < static_cast<size_t>(3 * v))
            return false;
        phi = block.phi0[static_cast<size_t>(local)];
        normal = Eigen::Vector3d(block.normal0[3 * static_cast<size_t>(local)],
                                 block.normal0[3 * static_cast<size_t>(local) + 1],
                                 block.normal0[3 * static_cast<size_t>(local) + 2]);
        if (hessian != nullptr)
        {
            if (!hasHessian || block.hessian0.size() < static_cast<size_t>(6 * v)) return false;
            const float* h = &block.hessian0[6 * static_cast<size_t>(local)];
            Eigen::Matrix3d& H = *hessian;
            H(0, 0) = h[0];
            H(0, 1) = H(1, 0) = h[1];
            H(0, 2) = H(2, 0) = h[2];
            H(1, 1) = h[3];
            H(1, 2) = H(2, 1) = h[4];
            H(2, 2) = h[5];
        }
        return true;
    }
};

} // namespace sdf
