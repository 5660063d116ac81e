// SdfOracle over libsdfo_cuda (plugins/SdfOracle/src/SdfOracle.cpp:152-444
// for the behaviour kept): the oracle owns its host data; its device copy is
// created on the first query and shared by copies of the oracle.  Every
// query mode runs on the GPU; results match the reference's queryFast to the
// FP32 storage / arithmetic tolerance (1e-5 relative).
#include "SdfOracle/SdfOracle.h"

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
    m_device->g = g;
    return g;
}

void SdfOracle::runQueries(const double* points, size_t n, QueryMode mode, float* gap,
                           float* normal, float* witness, unsigned char* valid) const
{
    const bool ca = m_sparse ? m_sparseData.hasContactCandidates() : m_data.hasContactCandidates();
    if (mode == QueryMode::ContactAware && ca)
        throw std::runtime_error("contact-aware candidate queries are not provided by the GPU backend");
    const sdfo_grid* g = deviceGrid();
    if (sdfo_query_host(g, modeId(mode), points, SDFO_POINTS_F64, static_cast<int64_t>(n), gap, nullptr,
                        normal, witness, valid, nullptr) != SDFO_OK)
        throw std::runtime_error(lastError());
}

SdfFastQueryResult SdfOracle::queryFast(const Eigen::Vector3d& point, QueryMode mode) const
{
    SdfFastQueryResult r;
    if (!isValid()) return r;
    float gap = 0.f, nrm[3], wit[3];
    unsigned char valid = 0;
    runQueries(point.data(), 1, mode, &gap, nrm, wit, &valid);
    r.valid = valid != 0;
    if (!r.valid) return r;
    r.gap = gap;
    r.gapNormal = Eigen::Vector3d(nrm[0], nrm[1], nrm[2]);
    r.witnessPoint = Eigen::Vector3d(wit[0], wit[1], wit[2]);
    r.candidateCount = 1;
    r.candidates[0] = SdfQueryCandidate{r.gap, r.gapNormal, r.witnessPoint, 0};
    return r;
}

SdfQueryResult SdfOracle::query(const Eigen::Vector3d& point, QueryMode mode) const
{
    const SdfFastQueryResult f = queryFast(point, mode);
    SdfQueryResult r;
    r.gap = f.gap;
    r.gapNormal = f.gapNormal;
    r.witnessPoint = f.witnessPoint;
    r.valid = f.valid;
    if (f.valid) r.candidates.push_back(f.candidates[0]);
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
    std::vector<float> gap(n), nrm(3 * n), wit(3 * n);
    std::vector<unsigned char> valid(n);
    runQueries(p.data(), n, mode, gap.data(), nrm.data(), wit.data(), valid.data());
    for (size_t i = 0; i < n; ++i)
    {
        SdfQueryResult& r = out[i];
        r.valid = valid[i] != 0;
        if (!r.valid) continue;
        r.gap = gap[i];
        r.gapNormal = Eigen::Vector3d(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]);
        r.witnessPoint = Eigen::Vector3d(wit[3 * i], wit[3 * i + 1], wit[3 * i + 2]);
        r.candidates.push_back(SdfQueryCandidate{r.gap, r.gapNormal, r.witnessPoint, 0});
    }
    return out;
}

} // namespace sdf
