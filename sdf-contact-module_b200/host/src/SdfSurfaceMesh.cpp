// Mesh file readers (formats of plugins/SdfOracle/src/SdfSurfaceMesh.cpp):
//  * OBJ: "v x y z" and "f a b c" (1-based; "a/b/c" forms keep the vertex
//    index), triangles only;
//  * NEXDYN_CONTACT_AWARE_SURFACE 1: named surfaces with an optional 4x4
//    row-major transform, "vertices N" + "v id x y z", "triangles M" +
//    "tri id v0 v1 v2" followed by three corner normals; "end" closes a
//    surface.  Vertices are transformed by the matrix, normals by its inverse
//    transpose and normalised.
#include "SdfOracle/SdfSurfaceMesh.h"

#include <cmath>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace sdf {
namespace {

std::string trimmed(std::string s)
{
    const size_t hash = s.find('#');
    if (hash != std::string::npos) s.erase(hash);
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return {};
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::runtime_error fail(const std::string& path, int line, const std::string& what)
{
    return std::runtime_error(path + ":" + std::to_string(line) + ": " + what);
}

struct Surface
{
    bool open{false};
    std::string name;
    int nVerts{-1}, nTris{-1}, seenVerts{0}, seenTris{0};
    Eigen::Matrix4d M{Eigen::Matrix4d::Identity()};
    Eigen::Matrix3d normalM{Eigen::Matrix3d::Identity()};
    std::unordered_map<int, int> ids;
};

void closeSurface(const std::string& path, int line, Surface& s)
{
    if (!s.open) return;
    if (s.nVerts < 0) throw fail(path, line, "surface '" + s.name + "' is missing vertices block");
    if (s.nTris < 0) throw fail(path, line, "surface '" + s.name + "' is missing triangles block");
    if (s.seenVerts != s.nVerts) throw fail(path, line, "surface '" + s.name + "' vertex count mismatch");
    if (s.seenTris != s.nTris) throw fail(path, line, "surface '" + s.name + "' triangle count mismatch");
    s = Surface{};
}

} // namespace

TriangleMesh loadObjFile(const std::string& path)
{
    std::ifstream ifs(path);
    if (!ifs.is_open()) throw std::runtime_error("Cannot open OBJ file: " + path);
    TriangleMesh mesh;
    std::string line;
    while (std::getline(ifs, line))
    {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream ss(line);
        std::string tok;
        ss >> tok;
        if (tok == "v")
        {
            double x = 0, y = 0, z = 0;
            ss >> x >> y >> z;
            mesh.vertices.emplace_back(x, y, z);
        }
        else if (tok == "f")
        {
            std::array<int, 3> t{};
            for (int c = 0; c < 3; ++c)
            {
                std::string f;
                ss >> f;
                t[static_cast<size_t>(c)] = std::stoi(f.substr(0, f.find('/'))) - 1;
            }
            mesh.triangles.push_back(t);
        }
    }
    return mesh;
}

CornerNormalTriangleMesh loadContactAwareSurfaceFile(const std::string& path)
{
    std::ifstream ifs(path);
    if (!ifs.is_open()) throw std::runtime_error("Cannot open contact-aware surface file: " + path);
    CornerNormalTriangleMesh mesh;
    Surface s;
    bool header = false;
    std::string raw;
    int lineNo = 0;
    while (std::getline(ifs, raw))
    {
        ++lineNo;
        const std::string line = trimmed(raw);
        if (line.empty()) continue;
        std::istringstream ss(line);
        std::string tok;
        ss >> tok;
        if (!header)
        {
            int version = 0;
            if (tok != "NEXDYN_CONTACT_AWARE_SURFACE" || !(ss >> version) || version != 1)
                throw fail(path, lineNo, "expected header 'NEXDYN_CONTACT_AWARE_SURFACE 1'");
            header = true;
            continue;
        }
        if (tok == "surface")
        {
            closeSurface(path, lineNo, s);
            s.open = true;
            if (!(ss >> s.name) || s.name.empty()) throw fail(path, lineNo, "surface requires a name");
            continue;
        }
        if (tok == "end")
        {
            closeSurface(path, lineNo, s);
            continue;
        }
        if (!s.open) throw fail(path, lineNo, "expected surface block");
        if (tok == "transform")
        {
            for (int r = 0; r < 4; ++r)
                for (int c = 0; c < 4; ++c)
                    if (!(ss >> s.M(r, c))) throw fail(path, lineNo, "transform requires 16 row-major values");
            const Eigen::Matrix3d L = s.M.block<3, 3>(0, 0);
            if (std::abs(L.determinant()) <= 1.0e-15)
                throw fail(path, lineNo, "transform linear part must be invertible");
            s.normalM = L.inverse().transpose();
        }
        else if (tok == "vertices")
        {
            if (!(ss >> s.nVerts) || s.nVerts < 0) throw fail(path, lineNo, "vertices requires a non-negative count");
        }
        else if (tok == "triangles")
        {
            if (!(ss >> s.nTris) || s.nTris < 0) throw fail(path, lineNo, "triangles requires a non-negative count");
        }
        else if (tok == "v")
        {
            if (s.nVerts < 0) throw fail(path, lineNo, "vertex appears before vertices block");
            int id = 0;
            Eigen::Vector3d p;
            if (!(ss >> id >> p.x() >> p.y() >> p.z())) throw fail(path, lineNo, "vertex requires: v <id> <x> <y> <z>");
            if (s.ids.count(id)) throw fail(path, lineNo, "duplicate vertex id in surface");
            s.ids.emplace(id, static_cast<int>(mesh.vertices.size()));
            const Eigen::Vector4d q = s.M * Eigen::Vector4d(p.x(), p.y(), p.z(), 1.0);
            mesh.vertices.push_back(std::abs(q.w()) > 1.0e-15 ? Eigen::Vector3d(q.head<3>() / q.w())
                                                              : Eigen::Vector3d(q.head<3>()));
            ++s.seenVerts;
        }
        else if (tok == "tri")
        {
            if (s.nTris < 0) throw fail(path, lineNo, "triangle appears before triangles block");
            int id = 0, v[3];
            Eigen::Vector3d n[3];
            if (!(ss >> id >> v[0] >> v[1] >> v[2] >> n[0].x() >> n[0].y() >> n[0].z() >> n[1].x() >>
                  n[1].y() >> n[1].z() >> n[2].x() >> n[2].y() >> n[2].z()))
                throw fail(path, lineNo, "triangle requires id, 3 vertex ids, and 3 corner normals");
            std::array<int, 3> t{};
            for (int c = 0; c < 3; ++c)
            {
                const auto it = s.ids.find(v[c]);
                if (it == s.ids.end()) throw fail(path, lineNo, "triangle references unknown vertex id");
                t[static_cast<size_t>(c)] = it->second;
                const Eigen::Vector3d m = s.normalM * n[c];
                const double len = m.norm();
                if (!m.allFinite() || !std::isfinite(len) || len <= 1.0e-15)
                    throw fail(path, lineNo, "corner normal must be a finite non-zero vector");
                n[c] = m / len;
            }
            const Eigen::Vector3d e0 = mesh.vertices[static_cast<size_t>(t[1])] - mesh.vertices[static_cast<size_t>(t[0])];
            const Eigen::Vector3d e1 = mesh.vertices[static_cast<size_t>(t[2])] - mesh.vertices[static_cast<size_t>(t[0])];
            if (e0.cross(e1).norm() <= 1.0e-15) throw fail(path, lineNo, "triangle is degenerate");
            mesh.triangles.push_back(t);
            mesh.cornerNormals.push_back({n[0], n[1], n[2]});
            ++s.seenTris;
        }
        else
        {
            throw fail(path, lineNo, "unknown token '" + tok + "'");
        }
    }
    if (!header) throw std::runtime_error(path + ": missing contact-aware surface header");
    closeSurface(path, lineNo, s);
    if (mesh.vertices.empty() || mesh.triangles.empty())
        throw std::runtime_error(path + ": contact-aware surface contains no triangles");
    return mesh;
}

} // namespace sdf
