// SdfOracle over libsdfo_cuda (plugins/SdfOracle/src/SdfOracle.cpp:152-444
// for the behaviour kept): the oracle owns its host data; its device copy is
// created on the first query and shared by copies of the oracle.  Every
// query mode runs on the GPU; results match the reference's queryFast to the
// FP32 storage / arithmetic tolerance (1e-5 relative); ContactAware queries
// on grids with candidates return the reference's candidate lists.
#include "SdfOracle/SdfOracle.h"

#include <algorithm>
#include <stdexcept>
#include <vector>

#include "SdfOracle/SdfIO.h"
#include "sdfo.h"

namespace sdf {
namespace {

std::string lastError()
{
    char buf[1024];
    sdfo_last_error(buf, sizeof(buf));
    return buf;
}

sdfo_grid_info infoFrom(const GridSpec& s)
{
    sdfo_grid_info info{};
    for (int a = 0; a < 3; ++a)
    {
        info.bmin[a] = s.bmin(a);
        info.bmax[a] = s.bmax(a);
        info.voxel[a] = s.voxel(a);
        info.shape[a] = s.shape[static_cast<size_t>(a)];
    }
    return info;
}

int32_t modeId(QueryMode m)
{
    switch (m)
    {
    case QueryMode::FirstOrder: return SDFO_FIRST_ORDER;
    case QueryMode::SecondOrder: return SDFO_SECOND_ORDER;
    case QueryMode::Trilinear: return SDFO_TRILINEAR;
    case QueryMode::Tricubic: return SDFO_TRICUBIC;
    case QueryMode::ContactAware: return SDFO_CONTACT_AWARE;
    }
    return SDFO_SECOND_ORDER;
}

} // namespace

struct SdfOracle::Device
{
    std::mutex m;
    sdfo_grid* g = nullptr;
    ~Device() { sdfo_grid_destroy(g); }
};

SdfOracle::SdfOracle(SdfData data) : m_data(std::move(data)), m_device(std::make_shared<Device>()) {}

SdfOracle::SdfOracle(SparseSdfData data)
    : m_sparseData(std::move(data)), m_sparse(true), m_device(std::make_shared<Device>())
{
}

SdfOracle SdfOracle::loadFromFile(const std::string& path)
{
    if (isSparseSdf(path)) return SdfOracle(loadSparseSdf(path));
    return SdfOracle(loadSdf(path));
}

const sdfo_grid* SdfOracle::deviceGrid() const
{
    if (!isValid() || !m_device) return nullptr;
    std::lock_guard<std::mutex> lock(m_device->m);
    if (m_device->g) return m_device->g;
    sdfo_grid* g = nullptr;
    int rc;
    if (!m_sparse)
    {
        const SdfData& d = m_data;
        const size_t N = static_cast<size_t>(d.spec.totalVoxels());
        std::vector<double> nrm(3 * N), hes(6 * N), wit(3 * N);
        for (size_t i = 0; i < N; ++i)
        {
            for (int a = 0; a < 3; ++a)
            {
                nrm[3 * i + static_cast<size_t>(a)] = d.n0[i](a);
                wit[3 * i + static_cast<size_t>(a)] = d.witness0[i](a);
            }
            const Eigen::Matrix3d& H = d.H0[i];
            const double v[6] = {H(0, 0), H(0, 1), H(0, 2), H(1, 1), H(1, 2), H(2, 2)};
            for (int q = 0; q < 6; ++q) hes[6 * i + static_cast<size_t>(q)] = v[q];
        }
        const sdfo_grid_info info = infoFrom(d.spec);
        rc = sdfo_grid_create_dense(&info, d.phi0.data(), nrm.data(), hes.data(), wit.data(), nullptr, &g);
    }
    else
    {
        const SparseSdfData& s = m_sparseData;
        const size_t B = s.blocks.size(), V = static_cast<size_t>(s.blockVoxelCount());
        std::vector<int32_t> ijk(3 * B);
        std::vector<float> phi(B * V), nrm(3 * B * V), hes(s.hasHessian ? 6 * B * V : 0);
        for (size_t b = 0; b < B; ++b)
        {
            const SparseSdfBlock& blk = s.blocks[b];
            for (int a = 0; a < 3; ++a) ijk[3 * b + static_cast<size_t>(a)] = blk.index[static_cast<size_t>(a)];
            std::copy(blk.phi0.begin(), blk.phi0.begin() + static_cast<long>(V), phi.begin() + static_cast<long>(b * V));
            std::copy(blk.normal0.begin(), blk.normal0.begin() + static_cast<long>(3 * V),
                      nrm.begin() + static_cast<long>(3 * b * V));
            if (s.hasHessian)
                std::copy(blk.hessian0.begin(), blk.hessian0.begin() + static_cast<long>(6 * V),
                          hes.begin() + static_cast<long>(6 * b * V));
        }
        sdfo_grid_info info = infoFrom(s.spec);
        info.block_dim = s.blockDim;
        info.halo_voxels = s.haloVoxels;
        info.block_count = static_cast<int32_t>(B);
        info.band_distance = s.bandDistance;
        rc = sdfo_grid_create_sparse(&info, ijk.data(), phi.data(), nrm.data(),
                                     s.hasHessian ? hes.data() : nullptr, nullptr, &g);
    }
    if (rc != SDFO_OK) throw std::runtime_error(lastError());
    // contact-aware candidates travel with the grid
    if (!m_sparse && m_data.hasContactCandidates())
    {
        const SdfData& d = m_data;
        std::vector<double> cn(3 * d.contactCandidateNormal0.size());
        for (size_t i = 0; i < d.contactCandidateNormal0.size(); ++i)
            for (int a = 0; a < 3; ++a) cn[3 * i + static_cast<size_t>(a)] = d.contactCandidateNormal0[i](a);
        rc = sdfo_grid_attach_candidates(g, d.contactCandidateStride, d.contactCandidateCount.data(),
                                         d.contactCandidatePhi0.data(), cn.data(),
                                         d.contactCandidateBranchId.data());
    }
    else if (m_sparse && m_sparseData.hasContactCandidates())
    {
        const SparseSdfData& sp = m_sparseData;
        const size_t V = static_cast<size_t>(sp.blockVoxelCount());
        const size_t S = static_cast<size_t>(sp.contactCandidateStride);
        std::vector<uint8_t> cnt;
        std::vector<double> ph, cn;
        std::vector<int32_t> br;
        for (const SparseSdfBlock& blk : sp.blocks)
        {
            cnt.insert(cnt.end(), blk.contactCandidateCount.begin(), blk.contactCandidateCount.begin() + static_cast<long>(V));
            for (size_t i = 0; i < V * S; ++i)
            {
                ph.push_back(blk.contactCandidatePhi0[i]);
                br.push_back(blk.contactCandidateBranchId[i]);
                for (int a = 0; a < 3; ++a) cn.push_back(blk.contactCandidateNormal0[3 * i + static_cast<size_t>(a)]);
            }
        }
        rc = sdfo_grid_attach_candidates(g, static_cast<int32_t>(S), cnt.data(), ph.data(), cn.data(), br.data());
    }
    if (rc != SDFO_OK)
    {
        const std::string err = lastError();
        sdfo_grid_destroy(g);
        throw std::runtime_error(err);
    }
    m_device->g = g;
    return g;
}

void SdfOracle::runQueries(const double* points, size_t n, QueryMode mode, float* gap,
                           float* normal, float* witness, unsigned char* valid) const
{
    const sdfo_grid* g = deviceGrid();
    if (sdfo_query_host(g, modeId(mode), points, SDFO_POINTS_F64, static_cast<int64_t>(n), gap, nullptr,
                        normal, witness, valid, nullptr) != SDFO_OK)
        throw std::runtime_error(lastError());
}

namespace {

// Per-point results with the candidate lists of SdfFastQueryResult.
struct CandidateBatch
{
    std::vector<float> gap, nrm, wit, kgap, kn, kw;
    std::vector<unsigned char> valid;
    std::vector<int32_t> ncand, kb;
    explicit CandidateBatch(size_t n)
        : gap(n), nrm(3 * n), wit(3 * n), kgap(8 * n), kn(24 * n), kw(24 * n), valid(n), ncand(n), kb(8 * n)
    {
    }
    SdfFastQueryResult at(size_t i) const
    {
        SdfFastQueryResult r;
        r.valid = valid[i] != 0;
        if (!r.valid) return r;
        r.gap = gap[i];
        r.gapNormal = Eigen::Vector3d(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
        r.witnessPoint = Eigen::Vector3d(wit[3 * i], wit[3 * i + 1], wit[3 * i + 2]);
        r.candidateCount = std::min(ncand[i], kMaxSdfQueryCandidates);
        for (int c = 0; c < r.candidateCount; ++c)
        {
            const size_t k = 8 * i + static_cast<size_t>(c);
            r.candidates[static_cast<size_t>(c)] = SdfQueryCandidate{
                kgap[k], Eigen::Vector3d(kn[3 * k], kn[3 * k + 1], kn[3 * k + 2]),
                Eigen::Vector3d(kw[3 * k], kw[3 * k + 1], kw[3 * k + 2]), kb[k]};
        }
        return r;
    }
};

void queryCandidates(const sdfo_grid* g, QueryMode mode, const double* pts, size_t n, CandidateBatch& b)
{
    if (sdfo_query_candidates_host(g, modeId(mode), pts, SDFO_POINTS_F64, static_cast<int64_t>(n),
                                   b.gap.data(), b.nrm.data(), b.wit.data(), b.valid.data(),
                                   b.ncand.data(), b.kgap.data(), b.kn.data(), b.kw.data(), b.kb.data(),
                                   nullptr) != SDFO_OK)
        throw std::runtime_error(lastError());
}

} // namespace

SdfFastQueryResult SdfOracle::queryFast(const Eigen::Vector3d& point, QueryMode mode) const
{
    if (!isValid()) return SdfFastQueryResult{};
    CandidateBatch b(1);
    queryCandidates(deviceGrid(), mode, point.data(), 1, b);
    return b.at(0);
}

SdfQueryResult SdfOracle::query(const Eigen::Vector3d& point, QueryMode mode) const
{
    const SdfFastQueryResult f = queryFast(point, mode);
    SdfQueryResult r;
    r.gap = f.gap;
    r.gapNormal = f.gapNormal;
    r.witnessPoint = f.witnessPoint;
    r.valid = f.valid;
    for (int c = 0; c < f.candidateCount; ++c) r.candidates.push_back(f.candidates[static_cast<size_t>(c)]);
    return r;
}

std::vector<SdfQueryResult> SdfOracle::queryBatch(const std::vector<Eigen::Vector3d>& points,
                                                  QueryMode mode) const
{
    const size_t n = points.size();
    std::vector<SdfQueryResult> out(n);
    if (!isValid() || n == 0) return out;
    std::vector<double> p(3 * n);
    for (size_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) p[3 * i + static_cast<size_t>(a)] = points[i](a);
    CandidateBatch b(n);
    queryCandidates(deviceGrid(), mode, p.data(), n, b);
    for (size_t i = 0; i < n; ++i)
    {
        const SdfFastQueryResult f = b.at(i);
        SdfQueryResult& r = out[i];
        r.valid = f.valid;
        if (!r.valid) continue;
        r.gap = f.gap;
        r.gapNormal = f.gapNormal;
        r.witnessPoint = f.witnessPoint;
        for (int c = 0; c < f.candidateCount; ++c) r.candidates.push_back(f.candidates[static_cast<size_t>(c)]);
    }
    return out;
}

} // namespace sdf
