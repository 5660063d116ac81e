#pragma once
// SDF queries (plugins/SdfOracle/include/SdfOracle/SdfOracle.h:11-67).  The
// oracle owns its SdfData / SparseSdfData like the reference and, on first
// use, a device copy in libsdfo_cuda; every query runs on the GPU.
// queryBatch issues one batched kernel for all points; query / queryFast are
// single-point calls of the same kernel (prefer queryBatch for throughput).
// A query before any grid is attached returns valid = false.

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "SdfOracle/SdfCommon.h"
#include "SdfOracle/SdfData.h"

struct sdfo_grid;

namespace sdf {

enum class QueryMode
{
    FirstOrder,
    SecondOrder,
    Trilinear,
    Tricubic,
    ContactAware
};

class SdfOracle
{
public:
    SdfOracle() = default;
    explicit SdfOracle(SdfData data);
    explicit SdfOracle(SparseSdfData data);

    static SdfOracle loadFromFile(const std::string& path);

    SdfQueryResult query(const Eigen::Vector3d& point,
                         QueryMode mode = QueryMode::SecondOrder) const;
    SdfFastQueryResult queryFast(const Eigen::Vector3d& point,
                                 QueryMode mode = QueryMode::SecondOrder) const;
    std::vector<SdfQueryResult> queryBatch(const std::vector<Eigen::Vector3d>& points,
                                           QueryMode mode = QueryMode::SecondOrder) const;

    const SdfData& data() const { return m_data; }
    const SparseSdfData& sparseData() const { return m_sparseData; }
    bool isSparse() const { return m_sparse; }
    const GridSpec& gridSpec() const { return m_sparse ? m_sparseData.spec : m_data.spec; }
    bool isValid() const { return m_sparse ? !m_sparseData.empty() : !m_data.phi0.empty(); }

    /// The device grid (created on first use); nullptr for an empty oracle.
    const sdfo_grid* deviceGrid() const;

private:
    struct Device;
    void runQueries(const double* points, size_t n, QueryMode mode, float* gap, float* normal,
                    float* witness, unsigned char* valid) const;

    SdfData m_data;
    SparseSdfData m_sparseData;
    bool m_sparse{false};
    std::shared_ptr<Device> m_device;
};

} // namespace sdf
