// Contact-aware SDF builds (SdfBuilder::buildContactAware /
// buildSparseContactAware, SdfBuilder.cpp:416-821): per voxel up to
// maxCandidates (<= 8) surface-feature candidates {phi, normal, branch id},
// the primary (smallest |phi|) also stored as the voxel's phi / n / witness.
//
// Device pipeline:
//   tile index   (buildContactTileIndex, SdfBuilder.cpp:202-243): one thread
//                per triangle counts the tiles its grown bounds overlap, a
//                scan places its (tile << 32 | triangle) keys, one radix sort
//                orders them by tile then triangle -- the reference's
//                per-tile lists in triangle order -- and a scan of the
//                per-tile counts gives the list offsets;
//   fill         one CTA per tile (dense) or per stored brick (sparse); the
//                voxels of a CTA walk the same triangle list in the same
//                order, so every triangle record is one broadcast load;
//                per voxel: the minimum distance over the list, the
//                candidates within minimum + tolerance merged by normal
//                angle, a stable sort by |phi| (buildContactCandidatesForPoint,
//                SdfBuilder.cpp:268-343), the reference tree's nearest
//                triangle as the fallback;
//   then the Hessian of the primary normals and, for sparse grids, block
//   activation from the tile lists (SdfBuilder.cpp:593-646) with the same
//   compaction as the plain sparse builder.
// This translation unit is compiled with -fmad=false: the FP64 expressions
// keep the reference's operation order, so every candidate (and the sort
// and merge decisions that depend on it) is bit-identical.
#include "build_common.cuh"

namespace sdfo {
namespace {

// Merged candidate groups kept per voxel: kCaFast in the fill kernels'
// thread-local lists; voxels with more groups (coarse grids where many
// differently oriented triangles lie within the tolerance) are finished by a
// second pass with lists of kCaWide entries in global scratch memory.
constexpr int kCaFast = 16;
constexpr int kCaWide = 512;
constexpr int kStatusCaOverflow = 2;

// One triangle of a contact-aware mesh (makeContactTriangleInfos,
// SdfBuilder.cpp:155-184): vertices, corner normals, face normal.
struct CaTri
{
    double a[3], b[3], c[3];
    double cn[9];
    double fn[3];
};

struct CaCand
{
    double phi, dist;
    d3 n, w;
    int branch;
};

__device__ __forceinline__ double norm3(const d3& v) { return sqrt(dot(v, v)); }

// normalizedOrDefault (SdfBuilder.cpp:27-43)
__device__ __forceinline__ d3 normalized_or(const d3& v, const d3& fb)
{
    const double n = norm3(v);
    if (n <= 1.0e-15)
    {
        const double f = norm3(fb);
        if (f > 1.0e-15) return mk(fb.x / f, fb.y / f, fb.z / f);
        return mk(1.0, 0.0, 0.0);
    }
    return mk(v.x / n, v.y / n, v.z / n);
}

// barycentricOnTriangle (SdfBuilder.cpp:45-67)
__device__ __forceinline__ d3 barycentric(const d3& p, const d3& a, const d3& b, const d3& c)
{
    const d3 v0 = sub(b, a), v1 = sub(c, a), v2 = sub(p, a);
    const double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1);
    const double d20 = dot(v2, v0), d21 = dot(v2, v1);
    const double denom = d00 * d11 - d01 * d01;
    if (fabs(denom) <= 1.0e-15) return mk(1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0);
    const double v = (d11 * d20 - d01 * d21) / denom;
    const double w = (d00 * d21 - d01 * d20) / denom;
    return mk(1.0 - v - w, v, w);
}

// branchIdFromNormal (SdfBuilder.cpp:114-134): FNV-1a over the normal's
// components quantised to 1/4095.
__device__ __forceinline__ int branch_id(const d3& raw)
{
    const d3 n = normalized_or(raw, mk(1.0, 0.0, 0.0));
    const double c[3] = {n.x, n.y, n.z};
    uint32_t hash = 2166136261u;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        const double v = fmax(-1.0, fmin(1.0, c[a]));
        hash ^= (uint32_t)(int32_t)llround(v * 4095.0);
        hash *= 16777619u;
    }
    return (int)(1u + (hash & 0x3fffffffu));
}

__device__ __forceinline__ d3 ld3(const double* p) { return mk(__ldg(p), __ldg(p + 1), __ldg(p + 2)); }

// (point - closest).norm() of makeContactCandidate, without the normal.
__device__ __forceinline__ double candidate_distance(const d3& p, const CaTri* t)
{
    const d3 cp = closest_point(p, ld3(t->a), ld3(t->b), ld3(t->c));
    return norm3(sub(p, cp));
}

// makeContactCandidate (SdfBuilder.cpp:245-266)
__device__ __forceinline__ void make_candidate(const d3& p, const CaTri* t, CaCand& out)
{
    const d3 a = ld3(t->a), b = ld3(t->b), c = ld3(t->c);
    const d3 cp = closest_point(p, a, b, c);
    const d3 bary = barycentric(cp, a, b, c);
    const d3 n0 = ld3(t->cn), n1 = ld3(t->cn + 3), n2 = ld3(t->cn + 6);
    const d3 raw = mk(bary.x * n0.x + bary.y * n1.x + bary.z * n2.x,
                      bary.x * n0.y + bary.y * n1.y + bary.z * n2.y,
                      bary.x * n0.z + bary.y * n1.z + bary.z * n2.z);
    out.n = normalized_or(raw, ld3(t->fn));
    const d3 d = sub(p, cp);
    out.phi = dot(d, out.n);
    out.dist = norm3(d);
    out.w = cp;
    out.branch = branch_id(out.n);
}

// buildContactCandidatesForPoint (SdfBuilder.cpp:268-343).  ids: the tile's
// list (NULL = all triangles); returns the merged candidate count before
// truncation (merged[] sorted by |phi|), or -1 when more than `cap` groups
// would be needed.  The reference sorts with std::sort, which for more than
// 16 elements does not keep the order of equal |phi|; the stable order used
// here differs from it only for exactly equal |phi| among more than 16
// groups.
template <class Tree>
__device__ int ca_point(const d3& p, const CaTri* __restrict__ tris, int nt,
                        const int* __restrict__ ids, int nids, const Tree& tree, double tol,
                        double cosMerge, CaCand* merged, int cap, int* status)
{
    // Pass 1: the nearest distance, and in tile order the triangles that can
    // pass the final filter dist <= minD + tol (a triangle within the running
    // minimum + tol when it is met: the running minimum never falls below the
    // final one, so every accepted triangle is listed).  Pass 2 then finishes
    // only the listed triangles, in the same order; a list that would
    // overflow falls back to finishing every triangle of the tile.
    constexpr int kList = 24;
    int list[kList];
    int nl = 0;
    bool list_over = false;
    double minD = DBL_MAX;
    for (int q = 0; q < nids; ++q)
    {
        const int t = ids ? __ldg(ids + q) : q;
        if (t < 0 || t >= nt) continue;
        const double d = candidate_distance(p, tris + t);
        minD = d < minD ? d : minD;
        if (d <= minD + tol)
        {
            if (nl < kList)
                list[nl++] = t;
            else
                list_over = true;
        }
    }
    int fallback = -1;
    if (!isfinite(minD))
    {
        const Nearest nb = tree_nearest(tree, p, status);
        fallback = nb.id;
        minD = nb.slot >= 0 ? sqrt(nb.sq) : DBL_MAX;
    }
    const double allowed = minD + tol;
    int nm = 0;
    bool over = false;
    auto try_tri = [&](int t) {
        if (over || t < 0 || t >= nt) return;
        CaCand c;
        make_candidate(p, tris + t, c);
        if (!(c.dist <= allowed)) return;
        // mergeContactCandidate (SdfBuilder.cpp:136-153)
        for (int e = 0; e < nm; ++e)
        {
            if (dot(merged[e].n, c.n) >= cosMerge)
            {
                if (fabs(c.phi) < fabs(merged[e].phi)) merged[e] = c;
                return;
            }
        }
        if (nm < cap)
            merged[nm++] = c;
        else
            over = true;
    };
    if (nids == 0)
        try_tri(fallback);
    else if (!list_over)
        for (int e = 0; e < nl; ++e) try_tri(list[e]);
    else
        for (int q = 0; q < nids; ++q)
        {
            const int t = ids ? __ldg(ids + q) : q;
            if (t < 0 || t >= nt || !(candidate_distance(p, tris + t) <= allowed)) continue;
            try_tri(t);
        }
    if (over) return -1;
    if (nm == 0)
    {
        if (fallback < 0) fallback = tree_nearest(tree, p, status).id;
        try_tri(fallback);
    }
    // stable insertion sort by |phi| (std::sort's own order for <= 16)
    for (int i = 1; i < nm; ++i)
    {
        const CaCand v = merged[i];
        int j = i;
        while (j > 0 && fabs(v.phi) < fabs(merged[j - 1].phi))
        {
            merged[j] = merged[j - 1];
            --j;
        }
        merged[j] = v;
    }
    return nm;
}

struct CaView
{
    const CaTri* tris;
    int nt;
    const int* tile_off; // ntiles + 1, or NULL without tile acceleration
    const int* tile_ids;
    int tile_dim, tnx, tny, tnz;
    double tol, cos_merge;
    int stride;
};

// ContactTileIndex::candidatesForVoxel (SdfBuilder.cpp:98-111)
__device__ __forceinline__ void voxel_list(const CaView& v, int i, int j, int k, const int*& ids,
                                           int& n)
{
    if (!v.tile_off)
    {
        ids = nullptr;
        n = v.nt;
        return;
    }
    const int ti = max(0, min(v.tnx - 1, i / v.tile_dim));
    const int tj = max(0, min(v.tny - 1, j / v.tile_dim));
    const int tk = max(0, min(v.tnz - 1, k / v.tile_dim));
    const int t = ti + v.tnx * (tj + v.tny * tk);
    const int a = __ldg(v.tile_off + t), b = __ldg(v.tile_off + t + 1);
    ids = v.tile_ids + a;
    n = b - a;
}

// Tiles overlapped by a triangle's bounds grown by `expansion`
// (buildContactTileIndex, SdfBuilder.cpp:217-241).
__device__ __forceinline__ void tri_tile_range(const CaTri& T, const SpecD& s, double expansion,
                                               int tile_dim, int lo[3], int hi[3])
{
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        const double A = T.a[a], B = T.b[a], C = T.c[a];
        double mn = B < A ? B : A;
        mn = C < mn ? C : mn;
        double mx = A < B ? B : A;
        mx = mx < C ? C : mx;
        const double l = mn - expansion, u = mx + expansion;
        int i0 = (int)floor((l - s.bmin[a]) / s.voxel[a] - 0.5);
        int i1 = (int)ceil((u - s.bmin[a]) / s.voxel[a] - 0.5);
        i0 = max(0, min(s.n[a] - 1, i0));
        i1 = max(0, min(s.n[a] - 1, i1));
        lo[a] = i0 / tile_dim;
        hi[a] = i1 / tile_dim;
    }
}

__global__ void k_ca_tile_count(const CaTri* __restrict__ tris, int nt, SpecD s, double expansion,
                                int tile_dim, int64_t* __restrict__ counts)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int lo[3], hi[3];
    tri_tile_range(tris[t], s, expansion, tile_dim, lo, hi);
    counts[t] = (int64_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
}

__global__ void k_ca_tile_emit(const CaTri* __restrict__ tris, int nt, SpecD s, double expansion,
                               int tile_dim, int tnx, int tny, const int64_t* __restrict__ offs,
                               uint64_t* __restrict__ keys, int* __restrict__ tile_count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    int lo[3], hi[3];
    tri_tile_range(tris[t], s, expansion, tile_dim, lo, hi);
    int64_t o = offs[t];
    for (int tk = lo[2]; tk <= hi[2]; ++tk)
        for (int tj = lo[1]; tj <= hi[1]; ++tj)
            for (int ti = lo[0]; ti <= hi[0]; ++ti)
            {
                const int tile = ti + tnx * (tj + tny * tk);
                keys[o++] = ((uint64_t)(uint32_t)tile << 32) | (uint32_t)t;
                atomicAdd(tile_count + tile, 1);
            }
}

__global__ void k_ca_tile_ids(const uint64_t* __restrict__ keys, int64_t n, int* __restrict__ ids)
{
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) ids[p] = (int)(uint32_t)(keys[p] & 0xffffffffu);
}

// Outputs of dense voxel idx from its sorted merged list (nm groups).
__device__ __forceinline__ void write_dense_voxel(int64_t idx, const CaCand* merged, int nm, int stride,
                                                  uint8_t* count, double* cphi, double* cn,
                                                  int32_t* cbr, double* phi64, double* n64,
                                                  double* w64, float4* phin)
{
    const int cnt = nm < stride ? nm : stride;
    count[idx] = (uint8_t)cnt;
    double p0 = 0.0;
    d3 n0 = mk(1.0, 0.0, 0.0), w0 = mk(0.0, 0.0, 0.0);
    if (cnt > 0)
    {
        p0 = merged[0].phi;
        n0 = merged[0].n;
        w0 = merged[0].w;
    }
    phi64[idx] = p0;
    n64[3 * idx] = n0.x;
    n64[3 * idx + 1] = n0.y;
    n64[3 * idx + 2] = n0.z;
    w64[3 * idx] = w0.x;
    w64[3 * idx + 1] = w0.y;
    w64[3 * idx + 2] = w0.z;
    phin[idx] = make_float4((float)p0, (float)n0.x, (float)n0.y, (float)n0.z);
    for (int q = 0; q < stride; ++q)
    {
        const int64_t o = idx * stride + q;
        const bool has = q < cnt;
        cphi[o] = has ? merged[q].phi : 0.0;
        cn[3 * o] = has ? merged[q].n.x : 1.0;
        cn[3 * o + 1] = has ? merged[q].n.y : 0.0;
        cn[3 * o + 2] = has ? merged[q].n.z : 0.0;
        cbr[o] = has ? merged[q].branch : -1;
    }
}

struct DenseOut
{
    uint8_t* count;
    double* cphi;
    double* cn;
    int32_t* cbr;
    double* phi64;
    double* n64;
    double* w64;
    float4* phin;
};

// Dense fill: one CTA per tile of tile_dim^3 voxels.  Voxels needing more
// than kCaFast groups go to the overflow list for the wide pass.
template <class Tree>
__global__ void __launch_bounds__(256)
    k_ca_dense_fill(CaView v, Tree tree, SpecD s, int tile_dim, int tnx, int tny, DenseOut out,
                    int64_t* __restrict__ over_list, unsigned long long* __restrict__ over_count,
                    int* status)
{
    const int tile = blockIdx.x;
    const int ti = tile % tnx, tj = (tile / tnx) % tny, tk = tile / (tnx * tny);
    const int V = tile_dim * tile_dim * tile_dim;
    CaCand merged[kCaFast];
    for (int l = threadIdx.x; l < V; l += blockDim.x)
    {
        const int i = ti * tile_dim + l % tile_dim;
        const int j = tj * tile_dim + (l / tile_dim) % tile_dim;
        const int k = tk * tile_dim + l / (tile_dim * tile_dim);
        if (i >= s.n[0] || j >= s.n[1] || k >= s.n[2]) continue;
        const int64_t idx = i + (int64_t)s.n[0] * (j + (int64_t)s.n[1] * k);
        const int* ids;
        int nids;
        voxel_list(v, i, j, k, ids, nids);
        const int nm = ca_point(voxel_center(s, i, j, k), v.tris, v.nt, ids, nids, tree, v.tol,
                                v.cos_merge, merged, kCaFast, status);
        if (nm < 0)
        {
            over_list[atomicAdd(over_count, 1ull)] = idx;
            continue;
        }
        write_dense_voxel(idx, merged, nm, v.stride, out.count, out.cphi, out.cn, out.cbr, out.phi64,
                          out.n64, out.w64, out.phin);
    }
}

// Wide pass over the overflow voxels: one thread each, kCaWide groups in
// global scratch (`scratch` + thread * kCaWide).
template <class Tree>
__global__ void __launch_bounds__(128)
    k_ca_dense_wide(CaView v, Tree tree, SpecD s, DenseOut out, const int64_t* __restrict__ list,
                    int64_t n, CaCand* __restrict__ scratch, int* status)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t idx = list[t];
    const int i = (int)(idx % s.n[0]), j = (int)((idx / s.n[0]) % s.n[1]),
              k = (int)(idx / ((int64_t)s.n[0] * s.n[1]));
    CaCand* merged = scratch + t * kCaWide;
    const int* ids;
    int nids;
    voxel_list(v, i, j, k, ids, nids);
    const int nm = ca_point(voxel_center(s, i, j, k), v.tris, v.nt, ids, nids, tree, v.tol,
                            v.cos_merge, merged, kCaWide, status);
    if (nm < 0)
    {
        atomicOr(status, kStatusCaOverflow);
        return;
    }
    write_dense_voxel(idx, merged, nm, v.stride, out.count, out.cphi, out.cn, out.cbr, out.phi64,
                      out.n64, out.w64, out.phin);
}

// Sparse block selection (SdfBuilder.cpp:593-646).
template <class Tree>
__global__ void k_ca_sparse_activate(CaView v, Tree tree, SpecD s, int bd, int nbx, int nby,
                                     int nbz, double activation, int32_t* __restrict__ flags,
                                     int* status)
{
    const int bl = blockIdx.x * blockDim.x + threadIdx.x;
    if (bl >= nbx * nby * nbz) return;
    const int bi = bl % nbx, bj = (bl / nbx) % nby, bk = bl / (nbx * nby);
    const int i0 = bi * bd, j0 = bj * bd, k0 = bk * bd;
    bool act = false;
    if (v.tile_off)
    {
        const int i1 = min(i0 + bd - 1, s.n[0] - 1), j1 = min(j0 + bd - 1, s.n[1] - 1),
                  k1 = min(k0 + bd - 1, s.n[2] - 1);
        for (int tk = k0 / v.tile_dim; tk <= k1 / v.tile_dim && !act; ++tk)
            for (int tj = j0 / v.tile_dim; tj <= j1 / v.tile_dim && !act; ++tj)
                for (int ti = i0 / v.tile_dim; ti <= i1 / v.tile_dim && !act; ++ti)
                {
                    const int t = ti + v.tnx * (tj + v.tny * tk);
                    act = __ldg(v.tile_off + t + 1) > __ldg(v.tile_off + t);
                }
    }
    else
    {
        const int i1 = min(i0 + bd, s.n[0]), j1 = min(j0 + bd, s.n[1]), k1 = min(k0 + bd, s.n[2]);
        const d3 c = mk(s.bmin[0] + s.voxel[0] * (0.5 * (double)(i0 + i1)),
                        s.bmin[1] + s.voxel[1] * (0.5 * (double)(j0 + j1)),
                        s.bmin[2] + s.voxel[2] * (0.5 * (double)(k0 + k1)));
        const double h = fmax(s.voxel[0], fmax(s.voxel[1], s.voxel[2]));
        const double blockRadius = 0.5 * sqrt(3.0) * (double)bd * h;
        const double limit = activation + blockRadius;
        // exact far-block reject, as block_active (build_common.cuh) argues:
        // nothing recorded below limit^2 (1 + 1e-9) means the full search's
        // distance is above the limit too
        if (tree_nearest(tree, c, status, nullptr, limit * limit * (1.0 + 1e-9)).slot >= 0)
        {
            const Nearest nb = tree_nearest(tree, c, status);
            const double dist = nb.slot >= 0 ? sqrt(nb.sq) : DBL_MAX;
            act = dist <= limit;
        }
    }
    flags[bl] = act ? 1 : 0;
}

struct SparseOut
{
    float4* phin;
    uint8_t* count;
    float* cphi;
    float* cn;
    int32_t* cbr;
};

__device__ __forceinline__ void write_sparse_voxel(int64_t vi, const CaCand* merged, int nm,
                                                   int stride, const SparseOut& out)
{
    const int cnt = nm < stride ? nm : stride;
    out.count[vi] = (uint8_t)cnt;
    out.phin[vi] = cnt > 0 ? make_float4((float)merged[0].phi, (float)merged[0].n.x,
                                         (float)merged[0].n.y, (float)merged[0].n.z)
                           : make_float4(0.f, 1.f, 0.f, 0.f);
    for (int q = 0; q < stride; ++q)
    {
        const int64_t o = vi * stride + q;
        const bool has = q < cnt;
        out.cphi[o] = has ? (float)merged[q].phi : 0.f;
        out.cn[3 * o] = has ? (float)merged[q].n.x : 0.f;
        out.cn[3 * o + 1] = has ? (float)merged[q].n.y : 0.f;
        out.cn[3 * o + 2] = has ? (float)merged[q].n.z : 0.f;
        out.cbr[o] = has ? merged[q].branch : -1;
    }
}

// Sparse brick fill: one CTA per stored block, FP32 storage; voxels needing
// more than kCaFast groups go to the overflow list.
template <class Tree>
__global__ void __launch_bounds__(256)
    k_ca_sparse_fill(CaView v, Tree tree, SpecD s, int bd, const int32_t* __restrict__ ijk,
                     SparseOut out, int64_t* __restrict__ over_list,
                     unsigned long long* __restrict__ over_count, int* status)
{
    const int blk = blockIdx.x;
    const int V = bd * bd * bd;
    const int bi = ijk[3 * blk], bj = ijk[3 * blk + 1], bk = ijk[3 * blk + 2];
    CaCand merged[kCaFast];
    for (int local = threadIdx.x; local < V; local += blockDim.x)
    {
        const int i = bi * bd + local % bd, j = bj * bd + (local / bd) % bd, k = bk * bd + local / (bd * bd);
        const int64_t vi = (int64_t)blk * V + local;
        int nm = 0;
        if (i < s.n[0] && j < s.n[1] && k < s.n[2])
        {
            const int* ids;
            int nids;
            voxel_list(v, i, j, k, ids, nids);
            nm = ca_point(voxel_center(s, i, j, k), v.tris, v.nt, ids, nids, tree, v.tol,
                          v.cos_merge, merged, kCaFast, status);
        }
        if (nm < 0)
        {
            over_list[atomicAdd(over_count, 1ull)] = vi;
            continue;
        }
        write_sparse_voxel(vi, merged, nm, v.stride, out);
    }
}

template <class Tree>
__global__ void __launch_bounds__(128)
    k_ca_sparse_wide(CaView v, Tree tree, SpecD s, int bd, const int32_t* __restrict__ ijk,
                     SparseOut out, const int64_t* __restrict__ list, int64_t n,
                     CaCand* __restrict__ scratch, int* status)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t vi = list[t];
    const int V = bd * bd * bd;
    const int blk = (int)(vi / V), local = (int)(vi % V);
    const int i = ijk[3 * blk] * bd + local % bd, j = ijk[3 * blk + 1] * bd + (local / bd) % bd,
              k = ijk[3 * blk + 2] * bd + local / (bd * bd);
    CaCand* merged = scratch + t * kCaWide;
    const int* ids;
    int nids;
    voxel_list(v, i, j, k, ids, nids);
    const int nm = ca_point(voxel_center(s, i, j, k), v.tris, v.nt, ids, nids, tree, v.tol,
                            v.cos_merge, merged, kCaWide, status);
    if (nm < 0)
    {
        atomicOr(status, kStatusCaOverflow);
        return;
    }
    write_sparse_voxel(vi, merged, nm, v.stride, out);
}

// Runs the wide pass over the overflow list in chunks whose scratch stays
// under about 256 MB.
template <class F>
void run_wide(const DeviceBuffer<int64_t>& list, const DeviceBuffer<unsigned long long>& count,
              cudaStream_t s, F&& launch)
{
    unsigned long long n = 0;
    SDFO_CUDA(cudaMemcpyAsync(&n, count.get(), sizeof(n), cudaMemcpyDeviceToHost, s));
    SDFO_CUDA(cudaStreamSynchronize(s));
    if (n == 0) return;
    const int64_t chunk = std::min<int64_t>((int64_t)n, 4096);
    DeviceBuffer<CaCand> scratch((size_t)chunk * kCaWide);
    for (int64_t a = 0; a < (int64_t)n; a += chunk)
    {
        const int64_t m = std::min<int64_t>(chunk, (int64_t)n - a);
        launch(list.get() + a, m, scratch.get());
        SDFO_CHECK_LAUNCH();
    }
    SDFO_CUDA(cudaStreamSynchronize(s));
}

// Host: triangle records (makeContactTriangleInfos) with the face normal
// normalizedOrDefault((b - a) x (c - a), UnitX).
std::vector<CaTri> make_tris(const double* verts, const int32_t* tris, int64_t nt,
                             const double* cnormals)
{
    std::vector<CaTri> out((size_t)nt);
    for (int64_t t = 0; t < nt; ++t)
    {
        CaTri& T = out[(size_t)t];
        for (int a = 0; a < 3; ++a)
        {
            T.a[a] = verts[3 * tris[3 * t] + a];
            T.b[a] = verts[3 * tris[3 * t + 1] + a];
            T.c[a] = verts[3 * tris[3 * t + 2] + a];
        }
        for (int q = 0; q < 9; ++q) T.cn[q] = cnormals[9 * t + q];
        const double e0[3] = {T.b[0] - T.a[0], T.b[1] - T.a[1], T.b[2] - T.a[2]};
        const double e1[3] = {T.c[0] - T.a[0], T.c[1] - T.a[1], T.c[2] - T.a[2]};
        const double cr[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2],
                              e0[0] * e1[1] - e0[1] * e1[0]};
        const double n = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
        if (n <= 1.0e-15)
        {
            T.fn[0] = 1.0;
            T.fn[1] = T.fn[2] = 0.0;
        }
        else
        {
            for (int a = 0; a < 3; ++a) T.fn[a] = cr[a] / n;
        }
    }
    return out;
}

// Device tile index (CSR): offsets over tnx*tny*tnz tiles, triangle ids in
// tile-then-triangle order.
struct TileIndex
{
    DeviceBuffer<int> off, ids;
    int tile_dim = 8, tnx = 1, tny = 1, tnz = 1;
};

void build_tile_index(TileIndex& ti, const CaTri* d_tris, int nt, const SpecD& s, int tile_dim,
                      double influence, cudaStream_t st)
{
    ti.tile_dim = std::max(1, tile_dim);
    ti.tnx = (s.n[0] + ti.tile_dim - 1) / ti.tile_dim;
    ti.tny = (s.n[1] + ti.tile_dim - 1) / ti.tile_dim;
    ti.tnz = (s.n[2] + ti.tile_dim - 1) / ti.tile_dim;
    const int ntiles = ti.tnx * ti.tny * ti.tnz;
    const double h = std::max({s.voxel[0], s.voxel[1], s.voxel[2]});
    const double tileRadius = 0.5 * std::sqrt(3.0) * (double)ti.tile_dim * h;
    volatile double ex = std::max(0.0, influence) + tileRadius;
    ex = ex + h;
    const double expansion = ex;
    const int T = 256;
    DeviceBuffer<int64_t> counts((size_t)nt + 1), offs((size_t)nt + 1);
    SDFO_CUDA(cudaMemsetAsync(counts.get(), 0, sizeof(int64_t) * (nt + 1), st));
    k_ca_tile_count<<<(nt + T - 1) / T, T, 0, st>>>(d_tris, nt, s, expansion, ti.tile_dim, counts.get());
    SDFO_CHECK_LAUNCH();
    size_t temp = 0;
    SDFO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, counts.get(), offs.get(), nt + 1, st));
    DeviceBuffer<unsigned char> tmp(temp);
    SDFO_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), temp, counts.get(), offs.get(), nt + 1, st));
    int64_t npairs = 0;
    SDFO_CUDA(cudaMemcpyAsync(&npairs, offs.get() + nt, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SDFO_CUDA(cudaStreamSynchronize(st));
    SDFO_REQUIRE(npairs < (int64_t(1) << 31), SDFO_ERR_INVALID_ARGUMENT,
                 "contact-aware tile index too large (more than 2^31 tile entries)");
    DeviceBuffer<uint64_t> keys((size_t)std::max<int64_t>(npairs, 1)),
        sorted((size_t)std::max<int64_t>(npairs, 1));
    DeviceBuffer<int> tile_count((size_t)ntiles + 1);
    SDFO_CUDA(cudaMemsetAsync(tile_count.get(), 0, sizeof(int) * (ntiles + 1), st));
    k_ca_tile_emit<<<(nt + T - 1) / T, T, 0, st>>>(d_tris, nt, s, expansion, ti.tile_dim, ti.tnx,
                                                    ti.tny, offs.get(), keys.get(), tile_count.get());
    SDFO_CHECK_LAUNCH();
    int end_bit = 32;
    while (end_bit < 64 && ((int64_t)1 << (end_bit - 32)) < ntiles) ++end_bit;
    if (npairs > 0)
    {
        size_t stemp = 0;
        SDFO_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, stemp, keys.get(), sorted.get(), (int)npairs,
                                                 0, end_bit, st));
        DeviceBuffer<unsigned char> stmp(stemp);
        SDFO_CUDA(cub::DeviceRadixSort::SortKeys(stmp.get(), stemp, keys.get(), sorted.get(),
                                                 (int)npairs, 0, end_bit, st));
        SDFO_CUDA(cudaStreamSynchronize(st));
    }
    ti.off.reset((size_t)ntiles + 1);
    size_t otemp = 0;
    SDFO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, otemp, tile_count.get(), ti.off.get(), ntiles + 1, st));
    DeviceBuffer<unsigned char> otmp(otemp);
    SDFO_CUDA(cub::DeviceScan::ExclusiveSum(otmp.get(), otemp, tile_count.get(), ti.off.get(),
                                            ntiles + 1, st));
    ti.ids.reset((size_t)std::max<int64_t>(npairs, 1));
    if (npairs > 0)
    {
        k_ca_tile_ids<<<(unsigned)((npairs + T - 1) / T), T, 0, st>>>(sorted.get(), npairs, ti.ids.get());
        SDFO_CHECK_LAUNCH();
    }
    SDFO_CUDA(cudaStreamSynchronize(st));
}

} // namespace

sdfo_grid* build_contact_aware(const double* verts, int64_t nv, const int32_t* tris, int64_t nt,
                               const double* cnormals, const sdfo_contact_aware_params& p,
                               cudaStream_t s)
{
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<sdfo_grid> g(new sdfo_grid());
    g->info = setup_grid(verts, nv, p.base);
    SDFO_CUDA(cudaGetDevice(&g->device));
    const SpecD sp = spec_of(g->info);
    const double h = std::max({g->info.voxel[0], g->info.voxel[1], g->info.voxel[2]});
    // SdfBuilder.cpp:450-456 / 563-569, 573-590
    const double tol = p.feature_distance_tolerance > 0.0 ? p.feature_distance_tolerance : 1.5 * h;
    const double cosMerge = std::cos(p.normal_merge_angle_degrees * std::acos(-1.0) / 180.0);
    const int stride = std::max(0, std::min(p.max_candidates, 8));
    const bool sparse = p.sparse != 0;
    const int bd = p.block_dim;
    const double band = p.band_distance > 0.0 ? p.band_distance : (double)p.band_voxels * h;
    volatile double actv = band + (double)p.halo_voxels * h;
    const double activation = actv;
    const double influence = sparse ? std::max(activation, tol + 2.0 * h) : tol + 2.0 * h;
    g->ca_stride = stride;
    g->info.candidate_stride = stride;
    g->stats.triangles = (int32_t)nt;
    g->stats.setup_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    Timer tm(s);
    AnyTree tree{bvh_mode()};
    tree.build(verts, nv, tris, nt, scene_extent(verts, nv, g->info), s);
    g->stats.bvh_nodes = tree.node_count(nt);
    const std::vector<CaTri> htris = make_tris(verts, tris, nt, cnormals);
    DeviceBuffer<CaTri> dtris((size_t)nt);
    SDFO_CUDA(cudaMemcpyAsync(dtris.get(), htris.data(), sizeof(CaTri) * nt, cudaMemcpyHostToDevice, s));
    TileIndex ti;
    if (p.use_tile_acceleration) build_tile_index(ti, dtris.get(), (int)nt, sp, p.tile_dim, influence, s);
    CaView v{};
    v.tris = dtris.get();
    v.nt = (int)nt;
    v.tile_off = p.use_tile_acceleration ? ti.off.get() : nullptr;
    v.tile_ids = p.use_tile_acceleration ? ti.ids.get() : nullptr;
    v.tile_dim = ti.tile_dim;
    v.tnx = ti.tnx;
    v.tny = ti.tny;
    v.tnz = ti.tnz;
    v.tol = tol;
    v.cos_merge = cosMerge;
    v.stride = stride;
    g->stats.bvh_ms = tm.lap();
    DeviceBuffer<int> status(1);
    SDFO_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), s));
    const int T = 256;
    if (!sparse)
    {
        const int64_t N = (int64_t)sp.n[0] * sp.n[1] * sp.n[2];
        g->stored_voxels = N;
        g->d.phin = dalloc<float4>((size_t)N);
        g->d.phi64 = dalloc<double>((size_t)N);
        g->d.n64 = dalloc<double>((size_t)N * 3);
        g->d.w64 = dalloc<double>((size_t)N * 3);
        g->d.h64 = dalloc<double>((size_t)N * 6);
        g->d.hess6 = dalloc<float>((size_t)N * 6);
        g->d.ca_count = dalloc<uint8_t>((size_t)N);
        g->d.ca_phi64 = dalloc<double>((size_t)N * std::max(stride, 1));
        g->d.ca_n64 = dalloc<double>((size_t)N * std::max(stride, 1) * 3);
        g->d.ca_branch = dalloc<int32_t>((size_t)N * std::max(stride, 1));
        // one CTA per fill tile (the tile index's tile edge, 8 without it)
        const int fd = p.use_tile_acceleration ? ti.tile_dim : 8;
        const int fx = (sp.n[0] + fd - 1) / fd, fy = (sp.n[1] + fd - 1) / fd, fz = (sp.n[2] + fd - 1) / fd;
        const DenseOut out{g->d.ca_count, g->d.ca_phi64, g->d.ca_n64, g->d.ca_branch,
                           g->d.phi64,    g->d.n64,      g->d.w64,  g->d.phin};
        DeviceBuffer<int64_t> over((size_t)N);
        DeviceBuffer<unsigned long long> over_n(1);
        SDFO_CUDA(cudaMemsetAsync(over_n.get(), 0, sizeof(unsigned long long), s));
        tree.visit([&](auto view) {
            k_ca_dense_fill<<<fx * fy * fz, T, 0, s>>>(v, view, sp, fd, fx, fy, out, over.get(),
                                                       over_n.get(), status.get());
            SDFO_CHECK_LAUNCH();
            run_wide(over, over_n, s, [&](const int64_t* list, int64_t m, CaCand* scratch) {
                k_ca_dense_wide<<<(unsigned)((m + 127) / 128), 128, 0, s>>>(v, view, sp, out, list, m,
                                                                          scratch, status.get());
            });
        });
        g->stats.fill_ms = tm.lap();
        g->info.has_hessian = 1;
        k_dense_hessian<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(sp, g->d.n64, g->d.h64, g->d.hess6);
        SDFO_CHECK_LAUNCH();
        if (!p.store_hessian)
        {
            // the reference leaves H0 at zero
            SDFO_CUDA(cudaMemsetAsync(g->d.h64, 0, sizeof(double) * 6 * N, s));
            SDFO_CUDA(cudaMemsetAsync(g->d.hess6, 0, sizeof(float) * 6 * N, s));
        }
        build_stencil_layouts(g.get(), s);
        g->stats.hessian_ms = tm.lap();
        g->stats.voxels_filled = N;
    }
    else
    {
        g->info.layout = SDFO_LAYOUT_SPARSE;
        g->info.block_dim = bd;
        g->info.halo_voxels = p.halo_voxels;
        g->info.band_distance = band;
        g->info.has_hessian = p.store_hessian ? 1 : 0;
        for (int a = 0; a < 3; ++a) g->nb[a] = (g->info.shape[a] + bd - 1) / bd;
        const int total = g->nb[0] * g->nb[1] * g->nb[2];
        g->stats.candidate_blocks = total;
        DeviceBuffer<int32_t> flags(total), slots(total);
        const int TA = spread_threads(total);
        tree.visit([&](auto view) {
            k_ca_sparse_activate<<<(total + TA - 1) / TA, TA, 0, s>>>(v, view, sp, bd, g->nb[0], g->nb[1],
                                                                  g->nb[2], activation, flags.get(),
                                                                  status.get());
        });
        SDFO_CHECK_LAUNCH();
        size_t temp = 0;
        SDFO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, flags.get(), slots.get(), total, s));
        DeviceBuffer<unsigned char> tmp(temp);
        SDFO_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), temp, flags.get(), slots.get(), total, s));
        int last_flag = 0, last_slot = 0;
        SDFO_CUDA(cudaMemcpyAsync(&last_flag, flags.get() + total - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        SDFO_CUDA(cudaMemcpyAsync(&last_slot, slots.get() + total - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        SDFO_CUDA(cudaStreamSynchronize(s));
        const int B = last_flag + last_slot;
        const int V = bd * bd * bd;
        g->info.block_count = B;
        g->stored_voxels = (int64_t)B * V;
        g->d.table = dalloc<int32_t>((size_t)total);
        g->d.ijk = dalloc<int32_t>((size_t)(B > 0 ? B : 1) * 3);
        k_sparse_table<<<(total + T - 1) / T, T, 0, s>>>(total, g->nb[0], g->nb[1], flags.get(),
                                                          slots.get(), g->d.table, g->d.ijk);
        SDFO_CHECK_LAUNCH();
        if (B > 0)
        {
            const int64_t NS = (int64_t)B * V;
            g->d.phin = dalloc<float4>((size_t)NS);
            g->d.ca_count = dalloc<uint8_t>((size_t)NS);
            g->d.ca_phi32 = dalloc<float>((size_t)NS * std::max(stride, 1));
            g->d.ca_n32 = dalloc<float>((size_t)NS * std::max(stride, 1) * 3);
            g->d.ca_branch = dalloc<int32_t>((size_t)NS * std::max(stride, 1));
            const SparseOut out{g->d.phin, g->d.ca_count, g->d.ca_phi32, g->d.ca_n32, g->d.ca_branch};
            DeviceBuffer<int64_t> over((size_t)NS);
            DeviceBuffer<unsigned long long> over_n(1);
            SDFO_CUDA(cudaMemsetAsync(over_n.get(), 0, sizeof(unsigned long long), s));
            tree.visit([&](auto view) {
                k_ca_sparse_fill<<<B, T, 0, s>>>(v, view, sp, bd, g->d.ijk, out, over.get(), over_n.get(),
                                                 status.get());
                SDFO_CHECK_LAUNCH();
                run_wide(over, over_n, s, [&](const int64_t* list, int64_t m, CaCand* scratch) {
                    k_ca_sparse_wide<<<(unsigned)((m + 127) / 128), 128, 0, s>>>(
                        v, view, sp, bd, g->d.ijk, out, list, m, scratch, status.get());
                });
            });
        }
        g->stats.fill_ms = tm.lap();
        if (B > 0 && p.store_hessian)
        {
            g->d.hess6 = dalloc<float>((size_t)B * V * 6);
            const int64_t stored = (int64_t)B * V;
            k_sparse_hessian<<<(unsigned)((stored + T - 1) / T), T, 0, s>>>(
                sp, bd, g->nb[0], g->nb[1], stored, g->d.ijk, g->d.table, g->d.phin, g->d.hess6);
            SDFO_CHECK_LAUNCH();
        }
        build_stencil_layouts(g.get(), s);
        g->stats.hessian_ms = tm.lap();
        g->stats.voxels_filled = (int64_t)B * V;
    }
    int hs = 0;
    SDFO_CUDA(cudaMemcpyAsync(&hs, status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SDFO_CUDA(cudaStreamSynchronize(s));
    if (hs & kStatusStackOverflow)
        throw Error(SDFO_ERR_DEVICE_STATUS, "BVH traversal stack overflow (tree deeper than 64)");
    if (hs & kStatusCaOverflow)
        throw Error(SDFO_ERR_UNSUPPORTED,
                    "contact-aware build: more than 512 merged candidate normals at a voxel");
    g->stats.total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return g.release();
}

} // namespace sdfo
