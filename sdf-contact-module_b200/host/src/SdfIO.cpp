// SDFO v0.1.0 reader / writer (byte layout: plugins/SdfOracle/src/
// SdfIO.cpp:60-552).  Errors are std::runtime_error with the reference's
// messages so callers that match on them keep working.
#include "SdfOracle/SdfIO.h"

#include <cstring>
#include <fstream>
#include <stdexcept>

namespace sdf {
namespace {

constexpr uint32_t kVersion = 100; // 0*10000 + 1*100 + 0
constexpr const char* kVersionString = "0.1.0";
constexpr uint32_t kFlagHessian = 1u, kFlagSparse = 2u, kFlagContactAware = 4u;
constexpr uint32_t kLayoutDense = 1u, kLayoutSparse = 2u, kLayoutDenseCA = 3u, kLayoutSparseCA = 4u;

// 128-byte header: magic, version, shape, bmin, bmax, voxel, flags, 32 bytes
// of layout-specific fields.
struct Header
{
    unsigned char raw[128];

    Header() { std::memset(raw, 0, sizeof(raw)); }

    template <class T>
    void put(int off, T v) { std::memcpy(raw + off, &v, sizeof(T)); }
    template <class T>
    T get(int off) const
    {
        T v;
        std::memcpy(&v, raw + off, sizeof(T));
        return v;
    }

    void setSpec(const GridSpec& s)
    {
        std::memcpy(raw, "SDFO", 4);
        put<uint32_t>(4, kVersion);
        for (int a = 0; a < 3; ++a)
        {
            put<uint32_t>(8 + 4 * a, static_cast<uint32_t>(s.shape[static_cast<size_t>(a)]));
            put<double>(20 + 8 * a, s.bmin(a));
            put<double>(44 + 8 * a, s.bmax(a));
            put<double>(68 + 8 * a, s.voxel(a));
        }
    }
    GridSpec spec() const
    {
        GridSpec s;
        for (int a = 0; a < 3; ++a)
        {
            s.shape[static_cast<size_t>(a)] = static_cast<int>(get<uint32_t>(8 + 4 * a));
            s.bmin(a) = get<double>(20 + 8 * a);
            s.bmax(a) = get<double>(44 + 8 * a);
            s.voxel(a) = get<double>(68 + 8 * a);
        }
        return s;
    }
    uint32_t flags() const { return get<uint32_t>(92); }
    uint32_t field(int off) const { return get<uint32_t>(96 + off); }
};

Header readHeader(std::ifstream& ifs, const std::string& path)
{
    if (!ifs.is_open()) throw std::runtime_error("Cannot open SdfOracle data file: " + path);
    Header h;
    ifs.read(reinterpret_cast<char*>(h.raw), sizeof(h.raw));
    if (ifs.gcount() != static_cast<std::streamsize>(sizeof(h.raw)))
        throw std::runtime_error("Failed to read SdfOracle data header");
    if (std::memcmp(h.raw, "SDFO", 4) != 0) throw std::runtime_error("Invalid SdfOracle data magic number");
    if (h.get<uint32_t>(4) != kVersion)
        throw std::runtime_error("Unsupported SdfOracle data version: " +
                                 std::to_string(h.get<uint32_t>(4)) + " (only " +
                                 std::string(kVersionString) + " is supported)");
    return h;
}

template <class T>
void writeN(std::ofstream& o, const T* p, size_t n)
{
    o.write(reinterpret_cast<const char*>(p), static_cast<std::streamsize>(n * sizeof(T)));
}
template <class T>
void readN(std::ifstream& i, T* p, size_t n)
{
    i.read(reinterpret_cast<char*>(p), static_cast<std::streamsize>(n * sizeof(T)));
}

} // namespace

bool saveSdf(const SdfData& data, const std::string& path)
{
    std::ofstream ofs(path, std::ios::binary);
    if (!ofs.is_open()) return false;
    const size_t N = static_cast<size_t>(data.spec.totalVoxels());
    const bool ca = data.hasContactCandidates();
    Header h;
    h.setSpec(data.spec);
    h.put<uint32_t>(92, kFlagHessian | (ca ? kFlagContactAware : 0u));
    h.put<uint32_t>(96, ca ? kLayoutDenseCA : kLayoutDense);
    if (ca) h.put<uint32_t>(100, static_cast<uint32_t>(data.contactCandidateStride));
    writeN(ofs, h.raw, sizeof(h.raw));
    writeN(ofs, data.phi0.data(), N);
    std::vector<double> buf(6 * N);
    for (size_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) buf[3 * i + static_cast<size_t>(a)] = data.n0[i](a);
    writeN(ofs, buf.data(), 3 * N);
    for (size_t i = 0; i < N; ++i)
    {
        const Eigen::Matrix3d& H = data.H0[i];
        const double v[6] = {H(0, 0), H(0, 1), H(0, 2), H(1, 1), H(1, 2), H(2, 2)};
        std::memcpy(&buf[6 * i], v, sizeof(v));
    }
    writeN(ofs, buf.data(), 6 * N);
    for (size_t i = 0; i < N; ++i)
        for (int a = 0; a < 3; ++a) buf[3 * i + static_cast<size_t>(a)] = data.witness0[i](a);
    writeN(ofs, buf.data(), 3 * N);
    if (ca)
    {
        std::vector<uint32_t> cnt(data.contactCandidateCount.begin(), data.contactCandidateCount.end());
        writeN(ofs, cnt.data(), cnt.size());
        writeN(ofs, data.contactCandidatePhi0.data(), data.contactCandidatePhi0.size());
        for (const Eigen::Vector3d& n : data.contactCandidateNormal0) writeN(ofs, n.data(), 3);
        writeN(ofs, data.contactCandidateBranchId.data(), data.contactCandidateBranchId.size());
    }
    return ofs.good();
}

SdfData loadSdf(const std::string& path)
{
    std::ifstream ifs(path, std::ios::binary);
    const Header h = readHeader(ifs, path);
    if (h.flags() & kFlagSparse)
        throw std::runtime_error("SdfOracle data file uses sparse layout; call loadSparseSdf");
    const uint32_t layout = h.field(0);
    if (layout != kLayoutDense && layout != kLayoutDenseCA)
        throw std::runtime_error("SdfOracle data file is not dense 0.1.0 layout");
    const bool caFlag = (h.flags() & kFlagContactAware) != 0;
    if ((layout == kLayoutDenseCA) != caFlag)
        throw std::runtime_error("Dense SDF 0.1.0 contact-aware flag/layout mismatch");
    SdfData d;
    d.resize(h.spec());
    const size_t N = static_cast<size_t>(d.spec.totalVoxels());
    readN(ifs, d.phi0.data(), N);
    std::vector<double> buf(6 * N);
    readN(ifs, buf.data(), 3 * N);
    for (size_t i = 0; i < N; ++i) d.n0[i] = Eigen::Vector3d(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
    if (h.flags() & kFlagHessian)
    {
        readN(ifs, buf.data(), 6 * N);
        for (size_t i = 0; i < N; ++i)
        {
            const double* v = &buf[6 * i];
            Eigen::Matrix3d& H = d.H0[i];
            H(0, 0) = v[0];
            H(0, 1) = H(1, 0) = v[1];
            H(0, 2) = H(2, 0) = v[2];
            H(1, 1) = v[3];
            H(1, 2) = H(2, 1) = v[4];
            H(2, 2) = v[5];
        }
    }
    readN(ifs, buf.data(), 3 * N);
    for (size_t i = 0; i < N; ++i)
        d.witness0[i] = Eigen::Vector3d(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
    if (caFlag)
    {
        const int stride = static_cast<int>(h.field(4));
        if (stride <= 0 || stride > SdfData::kMaxContactCandidates)
            throw std::runtime_error("Invalid contact-aware candidate stride");
        d.resizeContactCandidates(stride);
        std::vector<uint32_t> cnt(N);
        readN(ifs, cnt.data(), N);
        for (size_t i = 0; i < N; ++i)
        {
            if (cnt[i] > static_cast<uint32_t>(stride))
                throw std::runtime_error("Invalid contact-aware candidate count");
            d.contactCandidateCount[i] = static_cast<uint8_t>(cnt[i]);
        }
        readN(ifs, d.contactCandidatePhi0.data(), d.contactCandidatePhi0.size());
        for (Eigen::Vector3d& n : d.contactCandidateNormal0) readN(ifs, n.data(), 3);
        readN(ifs, d.contactCandidateBranchId.data(), d.contactCandidateBranchId.size());
    }
    if (!ifs) throw std::runtime_error("Failed to read dense SDF payload");
    return d;
}

bool saveSparseSdf(const SparseSdfData& data, const std::string& path)
{
    std::ofstream ofs(path, std::ios::binary);
    if (!ofs.is_open()) return false;
    const int V = data.blockVoxelCount();
    if (data.blockDim <= 0 || V <= 0) return false;
    const bool ca = data.hasContactCandidates();
    Header h;
    h.setSpec(data.spec);
    h.put<uint32_t>(92, kFlagSparse | (data.hasHessian ? kFlagHessian : 0u) | (ca ? kFlagContactAware : 0u));
    h.put<uint32_t>(96, ca ? kLayoutSparseCA : kLayoutSparse);
    h.put<uint32_t>(100, static_cast<uint32_t>(data.blockDim));
    h.put<uint32_t>(104, static_cast<uint32_t>(data.haloVoxels));
    h.put<uint32_t>(108, static_cast<uint32_t>(data.blocks.size()));
    h.put<double>(112, data.bandDistance);
    if (ca) h.put<uint32_t>(120, static_cast<uint32_t>(data.contactCandidateStride));
    writeN(ofs, h.raw, sizeof(h.raw));
    const size_t v = static_cast<size_t>(V), s = static_cast<size_t>(data.contactCandidateStride);
    for (const SparseSdfBlock& b : data.blocks)
    {
        if (b.phi0.size() < v || b.normal0.size() < 3 * v ||
            (data.hasHessian && b.hessian0.size() < 6 * v) ||
            (ca && !b.hasContactCandidates(V, data.contactCandidateStride)))
            return false;
        const int32_t hdr[4] = {b.index[0], b.index[1], b.index[2], 0};
        writeN(ofs, hdr, 4);
        writeN(ofs, b.phi0.data(), v);
        writeN(ofs, b.normal0.data(), 3 * v);
        if (data.hasHessian) writeN(ofs, b.hessian0.data(), 6 * v);
        if (ca)
        {
            writeN(ofs, b.contactCandidateCount.data(), v);
            writeN(ofs, b.contactCandidatePhi0.data(), v * s);
            writeN(ofs, b.contactCandidateNormal0.data(), 3 * v * s);
            writeN(ofs, b.contactCandidateBranchId.data(), v * s);
        }
    }
    return ofs.good();
}

SparseSdfData loadSparseSdf(const std::string& path)
{
    std::ifstream ifs(path, std::ios::binary);
    const Header h = readHeader(ifs, path);
    const uint32_t layout = h.field(0);
    const bool caFlag = (h.flags() & kFlagContactAware) != 0;
    if ((layout == kLayoutSparseCA) != caFlag)
        throw std::runtime_error("Sparse SDF 0.1.0 contact-aware flag/layout mismatch");
    const bool ca = caFlag && layout == kLayoutSparseCA;
    if ((h.flags() & kFlagSparse) == 0 || !(layout == kLayoutSparse || ca))
        throw std::runtime_error("SdfOracle data file is not sparse block 0.1.0");
    SparseSdfData d;
    d.spec = h.spec();
    d.blockDim = static_cast<int>(h.field(4));
    d.haloVoxels = static_cast<int>(h.field(8));
    const uint32_t count = h.field(12);
    d.bandDistance = h.get<double>(112);
    d.hasHessian = (h.flags() & kFlagHessian) != 0;
    d.contactCandidateStride = ca ? static_cast<int>(h.field(24)) : 0;
    if (d.blockDim <= 0) throw std::runtime_error("Sparse SDF blockDim must be positive");
    if (ca && (d.contactCandidateStride <= 0 || d.contactCandidateStride > SdfData::kMaxContactCandidates))
        throw std::runtime_error("Invalid sparse contact-aware candidate stride");
    const size_t v = static_cast<size_t>(d.blockVoxelCount()), s = static_cast<size_t>(d.contactCandidateStride);
    d.blocks.reserve(count);
    for (uint32_t b = 0; b < count; ++b)
    {
        int32_t hdr[4];
        readN(ifs, hdr, 4);
        if (!ifs) throw std::runtime_error("Failed to read sparse SDF block header");
        SparseSdfBlock blk;
        blk.index = {hdr[0], hdr[1], hdr[2]};
        blk.phi0.resize(v);
        blk.normal0.resize(3 * v);
        readN(ifs, blk.phi0.data(), v);
        readN(ifs, blk.normal0.data(), 3 * v);
        if (d.hasHessian)
        {
            blk.hessian0.resize(6 * v);
            readN(ifs, blk.hessian0.data(), 6 * v);
        }
        if (ca)
        {
            blk.contactCandidateCount.resize(v);
            blk.contactCandidatePhi0.resize(v * s);
            blk.contactCandidateNormal0.resize(3 * v * s);
            blk.contactCandidateBranchId.resize(v * s);
            readN(ifs, blk.contactCandidateCount.data(), v);
            readN(ifs, blk.contactCandidatePhi0.data(), v * s);
            readN(ifs, blk.contactCandidateNormal0.data(), 3 * v * s);
            readN(ifs, blk.contactCandidateBranchId.data(), v * s);
            for (uint8_t c : blk.contactCandidateCount)
                if (c > d.contactCandidateStride)
                    throw std::runtime_error("Invalid sparse contact-aware candidate count");
        }
        if (!ifs) throw std::runtime_error("Failed to read sparse SDF block payload");
        d.blocks.push_back(std::move(blk));
    }
    d.rebuildIndex();
    return d;
}

bool isValidSdf(const std::string& path)
{
    std::ifstream ifs(path, std::ios::binary);
    if (!ifs.is_open()) return false;
    Header h;
    ifs.read(reinterpret_cast<char*>(h.raw), sizeof(h.raw));
    return ifs.gcount() == static_cast<std::streamsize>(sizeof(h.raw)) &&
           std::memcmp(h.raw, "SDFO", 4) == 0 && h.get<uint32_t>(4) == kVersion;
}

bool isSparseSdf(const std::string& path)
{
    if (!isValidSdf(path)) return false;
    std::ifstream ifs(path, std::ios::binary);
    Header h;
    ifs.read(reinterpret_cast<char*>(h.raw), sizeof(h.raw));
    const uint32_t layout = h.field(0);
    return (h.flags() & kFlagSparse) != 0 && (layout == kLayoutSparse || layout == kLayoutSparseCA);
}

} // namespace sdf
