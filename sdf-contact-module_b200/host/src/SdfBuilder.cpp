// SdfBuilder over libsdfo_cuda: the grid is built on the GPU and exported
// into the plugin's host containers (SdfData FP64 / SparseSdfData FP32), so
// callers receive exactly what the reference builder returns
// (plugins/SdfOracle/src/SdfBuilder.cpp:364-407, 823-983).
#include "SdfOracle/SdfBuilder.h"

#include <algorithm>
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

// The dense grid of a handle as the reference's SdfData (FP64 arrays), with
// its contact-aware candidates when it has them.
SdfData toDense(const sdfo_grid* g)
{
    sdfo_grid_info info;
    sdfo_grid_get_info(g, &info);
    SdfData data;
    data.resize(toSpec(info));
    const size_t N = static_cast<size_t>(data.spec.totalVoxels());
    std::vector<double> nrm(3 * N), hes(6 * N), wit(3 * N);
    if (sdfo_grid_export_dense(g, data.phi0.data(), nrm.data(), hes.data(), wit.data()) != SDFO_OK)
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
    if (info.candidate_stride > 0)
    {
        data.resizeContactCandidates(info.candidate_stride);
        const size_t M = N * static_cast<size_t>(info.candidate_stride);
        std::vector<double> cn(3 * M);
        if (sdfo_grid_export_candidates(g, data.contactCandidateCount.data(),
                                        data.contactCandidatePhi0.data(), cn.data(),
                                        data.contactCandidateBranchId.data()) != SDFO_OK)
            throw std::runtime_error(lastError());
        for (size_t i = 0; i < M; ++i)
            data.contactCandidateNormal0[i] = Eigen::Vector3d(cn[3 * i], cn[3 * i + 1], cn[3 * i + 2]);
    }
    return data;
}

// The sparse grid of a handle as the reference's SparseSdfData (FP32
// blocks in stored order), with its contact-aware candidates.
SparseSdfData toSparse(const sdfo_grid* g)
{
    sdfo_grid_info info;
    sdfo_grid_get_info(g, &info);
    SparseSdfData s;
    s.spec = toSpec(info);
    s.blockDim = info.block_dim;
    s.haloVoxels = info.halo_voxels;
    s.bandDistance = info.band_distance;
    s.hasHessian = info.has_hessian != 0;
    const size_t B = static_cast<size_t>(info.block_count), V = static_cast<size_t>(s.blockVoxelCount());
    std::vector<int32_t> ijk(3 * B);
    std::vector<float> phi(B * V), nrm(3 * B * V), hes(s.hasHessian ? 6 * B * V : 0);
    if (B > 0 && sdfo_grid_export_sparse(g, ijk.data(), phi.data(), nrm.data(),
                                         s.hasHessian ? hes.data() : nullptr) != SDFO_OK)
        throw std::runtime_error(lastError());
    const size_t S = static_cast<size_t>(std::max(0, info.candidate_stride));
    std::vector<uint8_t> ccount(S ? B * V : 0);
    std::vector<double> cphi(S * B * V), cn(3 * S * B * V);
    std::vector<int32_t> cbr(S * B * V);
    if (S && B > 0 &&
        sdfo_grid_export_candidates(g, ccount.data(), cphi.data(), cn.data(), cbr.data()) != SDFO_OK)
        throw std::runtime_error(lastError());
    s.contactCandidateStride = static_cast<int>(S);
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
        if (S)
        {
            blk.contactCandidateCount.assign(ccount.begin() + static_cast<long>(b * V),
                                             ccount.begin() + static_cast<long>((b + 1) * V));
            blk.contactCandidatePhi0.resize(V * S);
            blk.contactCandidateNormal0.resize(3 * V * S);
            blk.contactCandidateBranchId.resize(V * S);
            for (size_t i = 0; i < V * S; ++i)
            {
                blk.contactCandidatePhi0[i] = static_cast<float>(cphi[b * V * S + i]);
                blk.contactCandidateBranchId[i] = cbr[b * V * S + i];
                for (int a = 0; a < 3; ++a)
                    blk.contactCandidateNormal0[3 * i + static_cast<size_t>(a)] =
                        static_cast<float>(cn[3 * (b * V * S + i) + static_cast<size_t>(a)]);
            }
        }
    }
    s.rebuildIndex();
    return s;
}

struct CaMesh
{
    HostMesh m;
    std::vector<double> cn;
};

CaMesh flattenCa(const CornerNormalTriangleMesh& mesh)
{
    CaMesh c{flatten(mesh.vertices, mesh.triangles), {}};
    c.cn.resize(9 * mesh.cornerNormals.size());
    for (size_t t = 0; t < mesh.cornerNormals.size(); ++t)
        for (size_t v = 0; v < 3; ++v)
            for (int a = 0; a < 3; ++a) c.cn[9 * t + 3 * v + static_cast<size_t>(a)] = mesh.cornerNormals[t][v](a);
    return c;
}

sdfo_contact_aware_params toCaParams(const ContactAwareBuilderParams& p, bool sparse)
{
    sdfo_contact_aware_params q;
    sdfo_contact_aware_params_default(&q);
    q.base = toParams(p);
    q.max_candidates = p.maxCandidates;
    q.tile_dim = p.tileDim;
    q.use_tile_acceleration = p.useTileAcceleration ? 1 : 0;
    q.store_hessian = p.storeHessian ? 1 : 0;
    q.feature_distance_tolerance = p.featureDistanceTolerance;
    q.normal_merge_angle_degrees = p.normalMergeAngleDegrees;
    q.sparse = sparse ? 1 : 0;
    q.block_dim = p.blockDim;
    q.halo_voxels = p.haloVoxels;
    q.band_voxels = p.bandVoxels;
    q.band_distance = p.bandDistance;
    return q;
}

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
    SdfData data = toDense(g.g);
    const size_t N = static_cast<size_t>(data.spec.totalVoxels());
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
    SparseSdfData s = toSparse(g.g);
    const size_t B = s.blocks.size();
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
    const CaMesh m = flattenCa(mesh);
    const sdfo_contact_aware_params p = toCaParams(params, false);
    GridGuard g;
    if (sdfo_grid_build_contact_aware(m.m.v.data(), static_cast<int64_t>(mesh.vertices.size()),
                                      m.m.t.data(), static_cast<int64_t>(mesh.triangles.size()),
                                      m.cn.data(), &p, nullptr, &g.g) != SDFO_OK)
        throw std::runtime_error(lastError());
    SdfData data = toDense(g.g);
    log(params, "[SdfBuilder] Contact-aware grid built on the GPU");
    return data;
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
    const CaMesh m = flattenCa(mesh);
    const sdfo_contact_aware_params p = toCaParams(params, true);
    GridGuard g;
    if (sdfo_grid_build_contact_aware(m.m.v.data(), static_cast<int64_t>(mesh.vertices.size()),
                                      m.m.t.data(), static_cast<int64_t>(mesh.triangles.size()),
                                      m.cn.data(), &p, nullptr, &g.g) != SDFO_OK)
        throw std::runtime_error(lastError());
    SparseSdfData s = toSparse(g.g);
    log(params, "[SdfBuilder] Sparse contact-aware SDF blocks: " + std::to_string(s.blocks.size()));
    return s;
}

} // namespace sdf
