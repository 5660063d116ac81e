// SdfBuilder over libsdfo_cuda: the grid is built on the GPU and exported
// into the plugin's host containers (SdfData FP64 / SparseSdfData FP32), so
// callers receive exactly what the reference builder returns
// (plugins/SdfOracle/src/SdfBuilder.cpp:364-407, 823-983).
#include "SdfOracle/SdfBuilder.h"

#include <chrono>
#include <stdexcept>
#include <string>
#include <vector>

#include "sdfo.h"

namespace sdf {
namespace {

std::string lastError()
{
    char buf[1024];
    sdfo_last_error(buf, sizeof(buf));
    return buf;
}

void log(const BuilderParams& p, const std::string& msg)
{
    if (p.logCallback) p.logCallback(msg);
}

struct HostMesh
{
    std::vector<double> v;
    std::vector<int32_t> t;
};

HostMesh flatten(const std::vector<Eigen::Vector3d>& vertices,
                 const std::vector<std::array<int, 3>>& triangles)
{
    HostMesh m;
    m.v.resize(3 * vertices.size());
    for (size_t i = 0; i < vertices.size(); ++i)
        for (int a = 0; a < 3; ++a) m.v[3 * i + static_cast<size_t>(a)] = vertices[i](a);
    m.t.resize(3 * triangles.size());
    for (size_t i = 0; i < triangles.size(); ++i)
        for (int a = 0; a < 3; ++a) m.t[3 * i + static_cast<size_t>(a)] = triangles[i][static_cast<size_t>(a)];
    return m;
}

sdfo_build_params toParams(const BuilderParams& p)
{
    sdfo_build_params q;
    q.padding = p.padding;
    q.voxel_size = p.voxelSize;
    q.target_resolution = p.targetResolution;
    q.max_resolution = p.maxResolution;
    return q;
}

GridSpec toSpec(const sdfo_grid_info& info)
{
    GridSpec s;
    for (int a = 0; a < 3; ++a)
    {
        s.bmin(a) = info.bmin[a];
        s.bmax(a) = info.bmax[a];
        s.voxel(a) = info.voxel[a];
        s.shape[static_cast<size_t>(a)] = info.shape[a];
    }
    return s;
}

struct GridGuard
{
    sdfo_grid* g = nullptr;
    ~GridGuard() { sdfo_grid_destroy(g); }
};

} // namespace

SdfData SdfBuilder::build(const std::vector<Eigen::Vector3d>& vertices,
                          const std::vector<std::array<int, 3>>& triangles,
                          const BuilderParams& params)
{
    if (vertices.empty() || triangles.empty())
        throw std::runtime_error("Empty mesh provided to SdfBuilder");
    const auto t0 = std::chrono::steady_clock::now();
    const HostMesh m = flatten(vertices, triangles);
    const sdfo_build_params p = toParams(params);
    GridGuard g;
    if (sdfo_grid_build_dense(m.v.data(), static_cast<int64_t>(vertices.size()), m.t.data(),
                              static_cast<int64_t>(triangles.size()), &p, nullptr, &g.g) != SDFO_OK)
        throw std::runtime_error(lastError());
    sdfo_grid_info info;
    sdfo_grid_get_info(g.g, &info);
    SdfData data;
    data.resize(toSpec(info));
    const size_t N = static_cast<size_t>(data.spec.totalVoxels());
    std::vector<double> nrm(3 * N), hes(6 * N), wit(3 * N);
    if (sdfo_grid_export_dense(g.g, data.phi0.data(), nrm.data(), hes.data(), wit.data()) != SDFO_OK)
        throw std::runtime_error(lastError());
    for (size_t i = 0; i < N; ++i)
    {
        data.n0[i] = Eigen::Vector3d(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
        data.witness0[i] = Eigen::Vector3d(wit[3 * i], wit[3 * i + 1], wit[3 * i + 2]);
        const double* h = &hes[6 * i];
        Eigen::Matrix3d& H = data.H0[i];
        H(0, 0) = h[0];
        H(0, 1) = H(1, 0) = h[1];
        H(0, 2) = H(2, 0) = h[2];
        H(1, 1) = h[3];
        H(1, 2) = H(2, 1) = h[4];
        H(2, 2) = h[5];
    }
    log(params, "[SdfBuilder] Grid: " + std::to_string(info.shape[0]) + " x " +
                    std::to_string(info.shape[1]) + " x " + std::to_string(info.shape[2]) + " = " +
                    std::to_string(N) + " voxels (GPU, " +
                    std::to_string(std::chrono::duration<double, std::milli>(
                                       std::chrono::steady_clock::now() - t0)
                                       .count()) +
                    " ms)");
    return data;
}

SdfData SdfBuilder::build(const TriangleMesh& mesh, const BuilderParams& params)
{
    return build(mesh.vertices, mesh.triangles, params);
}

SparseSdfData SdfBuilder::buildSparse(const std::vector<Eigen::Vector3d>& vertices,
                                      const std::vector<std::array<int, 3>>& triangles,
                                      const SparseBuilderParams& params)
{
    if (vertices.empty() || triangles.empty())
        throw std::runtime_error("Empty mesh provided to SdfBuilder");
    if (params.blockDim <= 0) throw std::runtime_error("Sparse SDF blockDim must be positive");
    const HostMesh m = flatten(vertices, triangles);
    sdfo_sparse_build_params p;
    p.base = toParams(params);
    p.block_dim = params.blockDim;
    p.halo_voxels = params.haloVoxels;
    p.band_voxels = params.bandVoxels;
    p.store_hessian = params.storeHessian ? 1 : 0;
    p.band_distance = params.bandDistance;
    GridGuard g;
    if (sdfo_grid_build_sparse(m.v.data(), static_cast<int64_t>(vertices.size()), m.t.data(),
                               static_cast<int64_t>(triangles.size()), &p, nullptr, &g.g) != SDFO_OK)
        throw std::runtime_error(lastError());
    sdfo_grid_info info;
    sdfo_grid_get_info(g.g, &info);
    SparseSdfData s;
    s.spec = toSpec(info);
    s.blockDim = info.block_dim;
    s.haloVoxels = info.halo_voxels;
    s.bandDistance = info.band_distance;
    s.hasHessian = info.has_hessian != 0;
    const size_t B = static_cast<size_t>(info.block_count), V = static_cast<size_t>(s.blockVoxelCount());
    std::vector<int32_t> ijk(3 * B);
    std::vector<float> phi(B * V), nrm(3 * B * V), hes(s.hasHessian ? 6 * B * V : 0);
    if (sdfo_grid_export_sparse(g.g, ijk.data(), phi.data(), nrm.data(),
                                s.hasHessian ? hes.data() : nullptr) != SDFO_OK)
        throw std::runtime_error(lastError());
    s.blocks.resize(B);
    for (size_t b = 0; b < B; ++b)
    {
        SparseSdfBlock& blk = s.blocks[b];
        blk.index = {ijk[3 * b], ijk[3 * b + 1], ijk[3 * b + 2]};
        blk.phi0.assign(phi.begin() + static_cast<long>(b * V), phi.begin() + static_cast<long>((b + 1) * V));
        blk.normal0.assign(nrm.begin() + static_cast<long>(3 * b * V),
                           nrm.begin() + static_cast<long>(3 * (b + 1) * V));
        if (s.hasHessian)
            blk.hessian0.assign(hes.begin() + static_cast<long>(6 * b * V),
                                hes.begin() + static_cast<long>(6 * (b + 1) * V));
    }
    s.rebuildIndex();
    log(params, "[SdfBuilder] Sparse SDF blocks: " + std::to_string(B));
    return s;
}

SparseSdfData SdfBuilder::buildSparse(const TriangleMesh& mesh, const SparseBuilderParams& params)
{
    return buildSparse(mesh.vertices, mesh.triangles, params);
}

SdfData SdfBuilder::buildContactAware(const CornerNormalTriangleMesh& mesh,
                                      const ContactAwareBuilderParams& params)
{
    if (mesh.vertices.empty() || mesh.triangles.empty())
        throw std::runtime_error("Empty mesh provided to contact-aware SdfBuilder");
    if (mesh.cornerNormals.size() != mesh.triangles.size())
        throw std::runtime_error("Contact-aware SDF requires one corner-normal triplet per triangle");
    if (params.maxCandidates <= 0)
        throw std::runtime_error("Contact-aware SDF maxCandidates must be positive");
    throw std::runtime_error("Contact-aware SDF builds are not provided by the GPU backend");
}

SparseSdfData SdfBuilder::buildSparseContactAware(const CornerNormalTriangleMesh& mesh,
                                                  const ContactAwareBuilderParams& params)
{
    if (mesh.vertices.empty() || mesh.triangles.empty())
        throw std::runtime_error("Empty mesh provided to sparse contact-aware SdfBuilder");
    if (mesh.cornerNormals.size() != mesh.triangles.size())
        throw std::runtime_error(
            "Sparse contact-aware SDF requires one corner-normal triplet per triangle");
    if (params.maxCandidates <= 0)
        throw std::runtime_error("Sparse contact-aware SDF maxCandidates must be positive");
    if (params.blockDim <= 0)
        throw std::runtime_error("Sparse contact-aware SDF blockDim must be positive");
    throw std::runtime_error("Contact-aware SDF builds are not provided by the GPU backend");
}

} // namespace sdf
