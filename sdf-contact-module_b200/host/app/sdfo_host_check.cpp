// Exercise of the C++ plugin API over the GPU backend, driven by
// tests/test_host_cpp.py:
//
//   sdfo_host_check io <in.sdf> <out.sdf>
//       loadSdf / loadSparseSdf then save again (byte-exact round trip).
//   sdfo_host_check build <mesh.obj> <res> <out_prefix> <points.bin>
//       loadObjFile, SdfBuilder::build + buildSparse (band 3), saveSdf /
//       saveSparseSdf, and SdfOracle::queryBatch of every mode on the points
//       (float64 x3 records) into <out_prefix>.q<mode>.<dense|sparse>.bin as
//       gap, normal(3), witness(3), valid per point (float64).
//   sdfo_host_check surface <in.ncas> <out.bin>
//       loadContactAwareSurfaceFile; writes nv, nt, vertices, triangles and
//       corner normals as float64.
//   sdfo_host_check ca <in.ncas> <res> <out_prefix> <points.bin>
//       SdfBuilder::buildContactAware + buildSparseContactAware (band 3),
//       saveSdf / saveSparseSdf, and SdfOracle::queryBatch in ContactAware
//       mode with the candidate lists into <out_prefix>.ca.<dense|sparse>.bin:
//       gap, normal(3), witness(3), valid, ncand, then 8 x (gap, normal(3),
//       witness(3), branch) per point (float64).
//   sdfo_host_check errors
//       the reference's exception messages for bad inputs.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "SdfOracle/NexDynAdapter.h"
#include "SdfOracle/SdfBuilder.h"
#include "SdfOracle/SdfIO.h"
#include "SdfOracle/SdfOracle.h"
#include "SdfOracle/SdfSurfaceMesh.h"

using namespace sdf;

static std::vector<Eigen::Vector3d> readPoints(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    std::vector<double> raw;
    double v;
    while (f.read(reinterpret_cast<char*>(&v), sizeof(v))) raw.push_back(v);
    std::vector<Eigen::Vector3d> pts(raw.size() / 3);
    for (size_t i = 0; i < pts.size(); ++i) pts[i] = Eigen::Vector3d(raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]);
    return pts;
}

static void writeResults(const std::string& path, const std::vector<SdfQueryResult>& r)
{
    std::ofstream f(path, std::ios::binary);
    for (const SdfQueryResult& q : r)
    {
        const double rec[8] = {q.gap, q.gapNormal.x(), q.gapNormal.y(), q.gapNormal.z(),
                               q.witnessPoint.x(), q.witnessPoint.y(), q.witnessPoint.z(),
                               q.valid ? 1.0 : 0.0};
        f.write(reinterpret_cast<const char*>(rec), sizeof(rec));
    }
}

static void writeCandidates(const std::string& path, const std::vector<SdfQueryResult>& r)
{
    std::ofstream f(path, std::ios::binary);
    for (const SdfQueryResult& q : r)
    {
        std::vector<double> rec = {q.gap, q.gapNormal.x(), q.gapNormal.y(), q.gapNormal.z(),
                                   q.witnessPoint.x(), q.witnessPoint.y(), q.witnessPoint.z(),
                                   q.valid ? 1.0 : 0.0, static_cast<double>(q.candidates.size())};
        for (size_t c = 0; c < 8; ++c)
        {
            if (c < q.candidates.size())
            {
                const SdfQueryCandidate& k = q.candidates[c];
                const double v[8] = {k.gap, k.gapNormal.x(), k.gapNormal.y(), k.gapNormal.z(),
                                     k.witnessPoint.x(), k.witnessPoint.y(), k.witnessPoint.z(),
                                     static_cast<double>(k.branchId)};
                rec.insert(rec.end(), v, v + 8);
            }
            else
            {
                rec.insert(rec.end(), 8, 0.0);
            }
        }
        f.write(reinterpret_cast<const char*>(rec.data()), static_cast<std::streamsize>(rec.size() * sizeof(double)));
    }
}

static int expectThrow(const char* what, const std::string& expected, void (*fn)())
{
    try
    {
        fn();
    }
    catch (const std::runtime_error& e)
    {
        if (expected == e.what()) return 0;
        std::cerr << what << ": got '" << e.what() << "'\n";
        return 1;
    }
    std::cerr << what << ": no exception\n";
    return 1;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const std::string cmd = argv[1];
    try
    {
        if (cmd == "io" && argc == 4)
        {
            if (!isValidSdf(argv[2])) return 3;
            if (isSparseSdf(argv[2]))
                return saveSparseSdf(loadSparseSdf(argv[2]), argv[3]) ? 0 : 4;
            return saveSdf(loadSdf(argv[2]), argv[3]) ? 0 : 4;
        }
        if (cmd == "build" && argc == 6)
        {
            const TriangleMesh mesh = loadObjFile(argv[2]);
            const int res = std::stoi(argv[3]);
            const std::string pre = argv[4];
            const std::vector<Eigen::Vector3d> pts = readPoints(argv[5]);
            BuilderParams p;
            p.targetResolution = p.maxResolution = res;
            SdfData dense = SdfBuilder::build(mesh, p);
            if (!saveSdf(dense, pre + ".dense.sdf")) return 5;
            SparseBuilderParams sp;
            sp.targetResolution = sp.maxResolution = res;
            sp.bandVoxels = 3;
            SparseSdfData sparse = SdfBuilder::buildSparse(mesh, sp);
            if (!saveSparseSdf(sparse, pre + ".sparse.sdf")) return 6;
            const StandaloneSdfOracle od(std::move(dense));
            const SdfOracle os(std::move(sparse));
            const QueryMode modes[4] = {QueryMode::FirstOrder, QueryMode::SecondOrder,
                                        QueryMode::Trilinear, QueryMode::Tricubic};
            for (int m = 0; m < 4; ++m)
            {
                writeResults(pre + ".q" + std::to_string(m) + ".dense.bin", od.queryBatch(pts, modes[m]));
                writeResults(pre + ".q" + std::to_string(m) + ".sparse.bin", os.queryBatch(pts, modes[m]));
            }
            // single-point paths agree with the batch
            const SdfQueryResult a = od.query(pts[0], QueryMode::Tricubic);
            const SdfFastQueryResult b = od.queryFast(pts[0], QueryMode::Tricubic);
            const SdfQueryResult c = od.queryBatch({pts[0]}, QueryMode::Tricubic)[0];
            if (a.valid != c.valid || a.gap != c.gap || b.gap != c.gap) return 7;
            if (a.valid && (a.candidates.size() != 1 || b.candidateCount != 1)) return 8;
            const SdfOracle empty;
            if (empty.query(pts[0]).valid || empty.isValid()) return 9;
            return 0;
        }
        if (cmd == "surface" && argc == 4)
        {
            const CornerNormalTriangleMesh m = loadContactAwareSurfaceFile(argv[2]);
            std::vector<double> out = {static_cast<double>(m.vertices.size()),
                                       static_cast<double>(m.triangles.size())};
            for (const auto& v : m.vertices) out.insert(out.end(), {v.x(), v.y(), v.z()});
            for (const auto& t : m.triangles)
                out.insert(out.end(), {double(t[0]), double(t[1]), double(t[2])});
            for (const auto& cn : m.cornerNormals)
                for (const auto& n : cn) out.insert(out.end(), {n.x(), n.y(), n.z()});
            std::ofstream f(argv[3], std::ios::binary);
            f.write(reinterpret_cast<const char*>(out.data()), static_cast<std::streamsize>(out.size() * sizeof(double)));
            return 0;
        }
        if (cmd == "ca" && argc == 6)
        {
            const CornerNormalTriangleMesh mesh = loadContactAwareSurfaceFile(argv[2]);
            const int res = std::stoi(argv[3]);
            const std::string pre = argv[4];
            const std::vector<Eigen::Vector3d> pts = readPoints(argv[5]);
            ContactAwareBuilderParams p;
            p.targetResolution = p.maxResolution = res;
            SdfData dense = SdfBuilder::buildContactAware(mesh, p);
            if (!saveSdf(dense, pre + ".ca_dense.sdf")) return 5;
            p.bandVoxels = 3;
            SparseSdfData sparse = SdfBuilder::buildSparseContactAware(mesh, p);
            if (!saveSparseSdf(sparse, pre + ".ca_sparse.sdf")) return 6;
            const SdfOracle od(std::move(dense));
            const SdfOracle os(std::move(sparse));
            writeCandidates(pre + ".ca.dense.bin", od.queryBatch(pts, QueryMode::ContactAware));
            writeCandidates(pre + ".ca.sparse.bin", os.queryBatch(pts, QueryMode::ContactAware));
            const SdfFastQueryResult f = od.queryFast(pts[0], QueryMode::ContactAware);
            const SdfQueryResult q = od.query(pts[0], QueryMode::ContactAware);
            if (f.valid != q.valid || f.gap != q.gap || f.candidateCount != static_cast<int>(q.candidates.size()))
                return 7;
            return 0;
        }
        if (cmd == "errors")
        {
            int bad = 0;
            bad += expectThrow("empty mesh", "Empty mesh provided to SdfBuilder",
                               [] { SdfBuilder::build(TriangleMesh{}); });
            bad += expectThrow("block dim", "Sparse SDF blockDim must be positive", [] {
                TriangleMesh m;
                m.vertices = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}};
                m.triangles = {{0, 1, 2}};
                SparseBuilderParams p;
                p.blockDim = 0;
                SdfBuilder::buildSparse(m, p);
            });
            bad += expectThrow("missing file", "Cannot open SdfOracle data file: /nonexistent.sdf",
                               [] { loadSdf("/nonexistent.sdf"); });
            bad += expectThrow("missing obj", "Cannot open OBJ file: /nonexistent.obj",
                               [] { loadObjFile("/nonexistent.obj"); });
            return bad;
        }
    }
    catch (const std::exception& e)
    {
        std::cerr << "error: " << e.what() << "\n";
        return 10;
    }
    return 2;
}
