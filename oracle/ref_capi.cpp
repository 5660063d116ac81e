// C wrapper around the reference SdfOracle C++ sources, for ctypes.
//
// Test infrastructure only.  oracle/Makefile compiles this file together with
// the reference's own plugins/SdfOracle/src/*.cpp (unmodified, where they lie)
// into oracle/_ref/libsdfo_ref.so.  Tests and the CPU baseline use it to
// (1) pin the oracle restatement in oracle/sdfo_port.c, (2) generate golden
// fixtures, and (3) time the reference's own OpenMP query/build loops.
//
// Wrapped reference entry points:
//   SdfBuilder::build / buildSparse           (src/SdfBuilder.cpp:364, 823)
//   SdfBuilder::buildContactAware / buildSparseContactAware (src/SdfBuilder.cpp:416, 551)
//   loadContactAwareSurfaceFile               (src/SdfSurfaceMesh.cpp:157)
//   SdfOracle::queryFast                      (src/SdfOracle.cpp:226)
//   saveSdf / loadSdf / saveSparseSdf / ...   (src/SdfIO.cpp:93-552)
//   KdTree::findSignedNearest                 (include/SdfOracle/KdTree.h:143)
#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include <omp.h>

#include "SdfOracle/KdTree.h"
#include "SdfOracle/SdfBuilder.h"
#include "SdfOracle/SdfIO.h"
#include "SdfOracle/SdfOracle.h"
#include "SdfOracle/SdfSurfaceMesh.h"

namespace {

thread_local std::string g_error;

struct RefHandle
{
    sdf::SdfOracle oracle;
};

std::vector<Eigen::Vector3d> toVerts(const double* v, int nv)
{
    std::vector<Eigen::Vector3d> out(static_cast<size_t>(nv));
    for (int i = 0; i < nv; ++i)
        out[static_cast<size_t>(i)] = Eigen::Vector3d(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    return out;
}

std::vector<std::array<int, 3>> toTris(const int* t, int nt)
{
    std::vector<std::array<int, 3>> out(static_cast<size_t>(nt));
    for (int i = 0; i < nt; ++i)
        out[static_cast<size_t>(i)] = {t[3 * i], t[3 * i + 1], t[3 * i + 2]};
    return out;
}

void quietLog(const std::string&) {}

} // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

void ref_set_threads(int n)
{
    if (n > 0) omp_set_num_threads(n);
}

int ref_max_threads() { return omp_get_max_threads(); }

void* ref_build_dense(const double* verts, int nv, const int* tris, int nt,
                      double padding, double voxelSize, int targetResolution,
                      int maxResolution, double* seconds)
{
    try
    {
        sdf::BuilderParams p;
        p.padding = padding;
        p.voxelSize = voxelSize;
        p.targetResolution = targetResolution;
        p.maxResolution = maxResolution;
        p.logCallback = quietLog;
        const auto vv = toVerts(verts, nv);
        const auto tt = toTris(tris, nt);
        const auto t0 = std::chrono::steady_clock::now();
        sdf::SdfData data = sdf::SdfBuilder::build(vv, tt, p);
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        auto* h = new RefHandle{sdf::SdfOracle(std::move(data))};
        return h;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return nullptr;
    }
}

void* ref_build_sparse(const double* verts, int nv, const int* tris, int nt,
                       double padding, double voxelSize, int targetResolution,
                       int maxResolution, int blockDim, int haloVoxels,
                       int bandVoxels, double bandDistance, int storeHessian,
                       double* seconds)
{
    try
    {
        sdf::SparseBuilderParams p;
        p.padding = padding;
        p.voxelSize = voxelSize;
        p.targetResolution = targetResolution;
        p.maxResolution = maxResolution;
        p.blockDim = blockDim;
        p.haloVoxels = haloVoxels;
        p.bandVoxels = bandVoxels;
        p.bandDistance = bandDistance;
        p.storeHessian = storeHessian != 0;
        p.logCallback = quietLog;
        const auto vv = toVerts(verts, nv);
        const auto tt = toTris(tris, nt);
        const auto t0 = std::chrono::steady_clock::now();
        sdf::SparseSdfData data = sdf::SdfBuilder::buildSparse(vv, tt, p);
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        auto* h = new RefHandle{sdf::SdfOracle(std::move(data))};
        return h;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return nullptr;
    }
}

void* ref_load(const char* path)
{
    try
    {
        auto* h = new RefHandle{sdf::SdfOracle::loadFromFile(path)};
        return h;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return nullptr;
    }
}

int ref_save(void* hp, const char* path)
{
    auto* h = static_cast<RefHandle*>(hp);
    if (h->oracle.isSparse()) return sdf::saveSparseSdf(h->oracle.sparseData(), path) ? 0 : -1;
    return sdf::saveSdf(h->oracle.data(), path) ? 0 : -1;
}

// kind 0: SdfOracle::loadFromFile; 1: loadSdf; 2: loadSparseSdf
// (SdfIO.cpp:277-523); *seconds = wall time of the load.
void* ref_load_kind(const char* path, int kind, double* seconds)
{
    try
    {
        const auto t0 = std::chrono::steady_clock::now();
        RefHandle* h = nullptr;
        if (kind == 1)
            h = new RefHandle{sdf::SdfOracle(sdf::loadSdf(path))};
        else if (kind == 2)
            h = new RefHandle{sdf::SdfOracle(sdf::loadSparseSdf(path))};
        else
            h = new RefHandle{sdf::SdfOracle::loadFromFile(path)};
        if (seconds)
            *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return h;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return nullptr;
    }
}

// saveSdf / saveSparseSdf with the wall time of the write.
int ref_save_timed(void* hp, const char* path, double* seconds)
{
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = ref_save(hp, path);
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}


void ref_free(void* hp) { delete static_cast<RefHandle*>(hp); }

// shape[3], bmin[3], bmax[3], voxel[3]; sparse: info[0]=blocks, info[1]=blockDim,
// info[2]=halo, info[3]=hasHessian; band[0]=bandDistance.
int ref_grid_info(void* hp, int* shape, double* bmin, double* bmax, double* voxel,
                  int* isSparse, int* info, double* band)
{
    auto* h = static_cast<RefHandle*>(hp);
    const sdf::GridSpec& s = h->oracle.gridSpec();
    for (int a = 0; a < 3; ++a)
    {
        shape[a] = s.shape[static_cast<size_t>(a)];
        bmin[a] = s.bmin(a);
        bmax[a] = s.bmax(a);
        voxel[a] = s.voxel(a);
    }
    *isSparse = h->oracle.isSparse() ? 1 : 0;
    if (h->oracle.isSparse())
    {
        const auto& sp = h->oracle.sparseData();
        info[0] = static_cast<int>(sp.blocks.size());
        info[1] = sp.blockDim;
        info[2] = sp.haloVoxels;
        info[3] = sp.hasHessian ? 1 : 0;
        band[0] = sp.bandDistance;
    }
    else
    {
        info[0] = info[1] = info[2] = 0;
        info[3] = 1;
        band[0] = 0.0;
    }
    return 0;
}

// Dense export: phi[N], normal[N*3], hessian6[N*6] (xx,xy,xz,yy,yz,zz), witness[N*3].
int ref_dense_export(void* hp, double* phi, double* normal, double* hessian6, double* witness)
{
    auto* h = static_cast<RefHandle*>(hp);
    if (h->oracle.isSparse()) return -1;
    const sdf::SdfData& d = h->oracle.data();
    const size_t n = d.phi0.size();
    for (size_t i = 0; i < n; ++i)
    {
        if (phi) phi[i] = d.phi0[i];
        if (normal)
            for (int a = 0; a < 3; ++a) normal[3 * i + a] = d.n0[i](a);
        if (witness)
            for (int a = 0; a < 3; ++a) witness[3 * i + a] = d.witness0[i](a);
        if (hessian6)
        {
            const auto& H = d.H0[i];
            hessian6[6 * i + 0] = H(0, 0);
            hessian6[6 * i + 1] = H(0, 1);
            hessian6[6 * i + 2] = H(0, 2);
            hessian6[6 * i + 3] = H(1, 1);
            hessian6[6 * i + 4] = H(1, 2);
            hessian6[6 * i + 5] = H(2, 2);
        }
    }
    return 0;
}

// Sparse export in stored block order: ijk[B*3], phi[B*V], normal[B*V*3], hessian6[B*V*6].
int ref_sparse_export(void* hp, int* ijk, float* phi, float* normal, float* hessian6)
{
    auto* h = static_cast<RefHandle*>(hp);
    if (!h->oracle.isSparse()) return -1;
    const auto& sp = h->oracle.sparseData();
    const size_t V = static_cast<size_t>(sp.blockVoxelCount());
    for (size_t b = 0; b < sp.blocks.size(); ++b)
    {
        const auto& blk = sp.blocks[b];
        for (int a = 0; a < 3; ++a) ijk[3 * b + static_cast<size_t>(a)] = blk.index[static_cast<size_t>(a)];
        if (phi) std::memcpy(phi + b * V, blk.phi0.data(), V * sizeof(float));
        if (normal) std::memcpy(normal + b * V * 3, blk.normal0.data(), 3 * V * sizeof(float));
        if (hessian6 && sp.hasHessian)
            std::memcpy(hessian6 + b * V * 6, blk.hessian0.data(), 6 * V * sizeof(float));
    }
    return 0;
}

// Batched queryFast (OpenMP static, as SdfOracleDemo.cpp:376-386 does).
// gap[n], normal[n*3], witness[n*3], valid[n].
int ref_query(void* hp, int mode, const double* pts, int64_t n, double* gap,
              double* normal, double* witness, unsigned char* valid)
{
    auto* h = static_cast<RefHandle*>(hp);
    const auto m = static_cast<sdf::QueryMode>(mode);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
    {
        const Eigen::Vector3d p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        const sdf::SdfFastQueryResult r = h->oracle.queryFast(p, m);
        if (gap) gap[i] = r.gap;
        for (int a = 0; a < 3; ++a)
        {
            if (normal) normal[3 * i + a] = r.gapNormal(a);
            if (witness) witness[3 * i + a] = r.witnessPoint(a);
        }
        if (valid) valid[i] = r.valid ? 1 : 0;
    }
    return 0;
}

// The demo's timed benchmark loop (SdfOracleDemo.cpp:373-386): returns seconds,
// valid count and mean |gap| over the valid queries.
double ref_query_bench(void* hp, int mode, const double* pts, int64_t n,
                       int64_t* validOut, double* avgAbsGap)
{
    auto* h = static_cast<RefHandle*>(hp);
    const auto m = static_cast<sdf::QueryMode>(mode);
    const auto t0 = std::chrono::steady_clock::now();
    int64_t valid = 0;
    double sumAbsGap = 0.0;
#pragma omp parallel for reduction(+ : valid, sumAbsGap) schedule(static)
    for (int64_t i = 0; i < n; ++i)
    {
        const Eigen::Vector3d p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        const sdf::SdfFastQueryResult r = h->oracle.queryFast(p, m);
        if (r.valid)
        {
            ++valid;
            sumAbsGap += std::abs(r.gap);
        }
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (validOut) *validOut = valid;
    if (avgAbsGap) *avgAbsGap = valid > 0 ? sumAbsGap / static_cast<double>(valid) : 0.0;
    return std::chrono::duration<double>(t1 - t0).count();
}

// KdTree::findSignedNearest for a batch of points: signed distance, closest
// point, face normal of the chosen triangle, and triangle index.
int ref_signed_nearest(const double* verts, int nv, const int* tris, int nt,
                       const double* pts, int64_t n, double* sd, double* cp,
                       double* fn, int* tri)
{
    try
    {
        const auto vv = toVerts(verts, nv);
        const auto tt = toTris(tris, nt);
        sdf::KdTree tree;
        tree.build(vv, tt);
#pragma omp parallel for schedule(dynamic, 256)
        for (int64_t i = 0; i < n; ++i)
        {
            const Eigen::Vector3d p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
            const auto r = tree.findSignedNearest(p);
            sd[i] = r.signedDistance;
            for (int a = 0; a < 3; ++a)
            {
                cp[3 * i + a] = r.closestPoint(a);
                fn[3 * i + a] = r.normal(a);
            }
            tri[i] = r.triangleIndex;
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return -1;
    }
}

// loadObjFile: returns counts; call twice (first with null buffers).
int ref_load_obj(const char* path, double* verts, int* nv, int* tris, int* nt)
{
    try
    {
        const sdf::TriangleMesh m = sdf::loadObjFile(path);
        if (verts)
            for (size_t i = 0; i < m.vertices.size(); ++i)
                for (int a = 0; a < 3; ++a) verts[3 * i + static_cast<size_t>(a)] = m.vertices[i](a);
        if (tris)
            for (size_t i = 0; i < m.triangles.size(); ++i)
                for (int a = 0; a < 3; ++a) tris[3 * i + static_cast<size_t>(a)] = m.triangles[i][static_cast<size_t>(a)];
        *nv = static_cast<int>(m.vertices.size());
        *nt = static_cast<int>(m.triangles.size());
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return -1;
    }
}


// SdfBuilder::buildContactAware / buildSparseContactAware (sparse != 0) on a
// mesh with corner normals (nt, 3, 3).
void* ref_build_contact_aware(const double* verts, int nv, const int* tris, int nt,
                              const double* cornerNormals, double padding, double voxelSize,
                              int targetResolution, int maxResolution, int maxCandidates,
                              double featureDistanceTolerance, double normalMergeAngleDegrees,
                              int tileDim, int useTileAcceleration, int storeHessian, int sparse,
                              int blockDim, int haloVoxels, int bandVoxels, double bandDistance,
                              double* seconds)
{
    try
    {
        sdf::ContactAwareBuilderParams p;
        p.padding = padding;
        p.voxelSize = voxelSize;
        p.targetResolution = targetResolution;
        p.maxResolution = maxResolution;
        p.maxCandidates = maxCandidates;
        p.featureDistanceTolerance = featureDistanceTolerance;
        p.normalMergeAngleDegrees = normalMergeAngleDegrees;
        p.tileDim = tileDim;
        p.useTileAcceleration = useTileAcceleration != 0;
        p.storeHessian = storeHessian != 0;
        p.sparse = sparse != 0;
        p.blockDim = blockDim;
        p.haloVoxels = haloVoxels;
        p.bandVoxels = bandVoxels;
        p.bandDistance = bandDistance;
        p.logCallback = quietLog;
        sdf::CornerNormalTriangleMesh mesh;
        mesh.vertices = toVerts(verts, nv);
        mesh.triangles = toTris(tris, nt);
        mesh.cornerNormals.resize(static_cast<size_t>(nt));
        for (int t = 0; t < nt; ++t)
            for (int v = 0; v < 3; ++v)
                mesh.cornerNormals[static_cast<size_t>(t)][static_cast<size_t>(v)] =
                    Eigen::Vector3d(cornerNormals[9 * t + 3 * v], cornerNormals[9 * t + 3 * v + 1],
                                    cornerNormals[9 * t + 3 * v + 2]);
        const auto t0 = std::chrono::steady_clock::now();
        RefHandle* h = nullptr;
        if (sparse)
            h = new RefHandle{sdf::SdfOracle(sdf::SdfBuilder::buildSparseContactAware(mesh, p))};
        else
            h = new RefHandle{sdf::SdfOracle(sdf::SdfBuilder::buildContactAware(mesh, p))};
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        return h;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return nullptr;
    }
}

// Candidate stride of a contact-aware grid (0 = none).
int ref_ca_stride(void* hp)
{
    auto* h = static_cast<RefHandle*>(hp);
    return h->oracle.isSparse() ? h->oracle.sparseData().contactCandidateStride
                                : h->oracle.data().contactCandidateStride;
}

// Dense candidates: count[N], phi[N*s], normal[N*s*3], branch[N*s].
int ref_ca_export_dense(void* hp, unsigned char* count, double* phi, double* normal, int* branch)
{
    auto* h = static_cast<RefHandle*>(hp);
    if (h->oracle.isSparse()) return -1;
    const sdf::SdfData& d = h->oracle.data();
    const size_t N = d.contactCandidateCount.size(), M = d.contactCandidatePhi0.size();
    std::memcpy(count, d.contactCandidateCount.data(), N);
    std::memcpy(phi, d.contactCandidatePhi0.data(), M * sizeof(double));
    for (size_t i = 0; i < M; ++i)
        for (int a = 0; a < 3; ++a) normal[3 * i + a] = d.contactCandidateNormal0[i](a);
    std::memcpy(branch, d.contactCandidateBranchId.data(), M * sizeof(int));
    return 0;
}

// Sparse candidates per block in stored order: count[B*V], phi[B*V*s],
// normal[B*V*s*3], branch[B*V*s].
int ref_ca_export_sparse(void* hp, unsigned char* count, float* phi, float* normal, int* branch)
{
    auto* h = static_cast<RefHandle*>(hp);
    if (!h->oracle.isSparse()) return -1;
    const sdf::SparseSdfData& sp = h->oracle.sparseData();
    const int V = sp.blockDim * sp.blockDim * sp.blockDim;
    const int s = sp.contactCandidateStride;
    for (size_t b = 0; b < sp.blocks.size(); ++b)
    {
        const auto& blk = sp.blocks[b];
        std::memcpy(count + b * V, blk.contactCandidateCount.data(), (size_t)V);
        std::memcpy(phi + b * V * s, blk.contactCandidatePhi0.data(), (size_t)V * s * sizeof(float));
        std::memcpy(normal + b * V * s * 3, blk.contactCandidateNormal0.data(),
                    (size_t)V * s * 3 * sizeof(float));
        std::memcpy(branch + b * V * s, blk.contactCandidateBranchId.data(), (size_t)V * s * sizeof(int));
    }
    return 0;
}

// queryFast with its candidate list: ncand[n], kgap[n*8], knormal[n*24],
// kwitness[n*24], kbranch[n*8] (plus gap/normal/witness/valid as ref_query).
int ref_query_candidates(void* hp, int mode, const double* pts, int64_t n, double* gap,
                         double* normal, double* witness, unsigned char* valid, int* ncand,
                         double* kgap, double* knormal, double* kwitness, int* kbranch)
{
    auto* h = static_cast<RefHandle*>(hp);
    const auto m = static_cast<sdf::QueryMode>(mode);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i)
    {
        const Eigen::Vector3d p(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        const sdf::SdfFastQueryResult r = h->oracle.queryFast(p, m);
        gap[i] = r.gap;
        valid[i] = r.valid ? 1 : 0;
        ncand[i] = r.candidateCount;
        for (int a = 0; a < 3; ++a)
        {
            normal[3 * i + a] = r.gapNormal(a);
            witness[3 * i + a] = r.witnessPoint(a);
        }
        for (int c = 0; c < 8; ++c)
        {
            const sdf::SdfQueryCandidate& k = r.candidates[static_cast<size_t>(c)];
            kgap[8 * i + c] = k.gap;
            kbranch[8 * i + c] = k.branchId;
            for (int a = 0; a < 3; ++a)
            {
                knormal[24 * i + 3 * c + a] = k.gapNormal(a);
                kwitness[24 * i + 3 * c + a] = k.witnessPoint(a);
            }
        }
    }
    return 0;
}

// loadContactAwareSurfaceFile: call with NULL arrays for the counts, then
// with arrays of those sizes (verts (nv,3), tris (nt,3), normals (nt,3,3)).
int ref_load_ca_surface(const char* path, double* verts, int* nv, int* tris, int* nt,
                        double* normals)
{
    try
    {
        const sdf::CornerNormalTriangleMesh m = sdf::loadContactAwareSurfaceFile(path);
        *nv = static_cast<int>(m.vertices.size());
        *nt = static_cast<int>(m.triangles.size());
        if (verts)
            for (size_t i = 0; i < m.vertices.size(); ++i)
                for (int a = 0; a < 3; ++a) verts[3 * i + a] = m.vertices[i](a);
        if (tris)
            for (size_t i = 0; i < m.triangles.size(); ++i)
                for (int a = 0; a < 3; ++a) tris[3 * i + a] = m.triangles[i][static_cast<size_t>(a)];
        if (normals)
            for (size_t i = 0; i < m.cornerNormals.size(); ++i)
                for (int v = 0; v < 3; ++v)
                    for (int a = 0; a < 3; ++a)
                        normals[9 * i + 3 * v + a] = m.cornerNormals[i][static_cast<size_t>(v)](a);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_error = e.what();
        return -1;
    }
}

} // extern "C"
