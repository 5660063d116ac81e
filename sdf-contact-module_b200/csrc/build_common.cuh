// Device building blocks of the SDF builders, shared by the single-mesh
// builders (build.cu) and the batched builder (batch.cu): FP64 triangle
// primitives in the reference's operation order, the LBVH and the
// reference-order tree with their traversals, and the fill / Hessian /
// activation kernels.  Every translation unit that includes this header is
// compiled with -fmad=false (FP64 expressions evaluated as written), which is
// what makes the builds bit-identical to the reference's FP64 arithmetic.
#pragma once

#include <cub/cub.cuh>

#include <algorithm>
#include <thread>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "sdfo_internal.cuh"

namespace sdfo {

namespace {

constexpr int kStackDepth = 64;
constexpr int kStatusStackOverflow = 1;

// ---------------------------------------------------------------------------
// FP64 triangle primitives, in the reference's operation order
// ---------------------------------------------------------------------------
struct d3
{
    double x, y, z;
};
__device__ __forceinline__ d3 mk(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ d3 sub(const d3& a, const d3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double dot(const d3& a, const d3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(const d3& a, const d3& b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Voronoi region of a closest point: the vertices a, b, c, the edges ab, ac,
// bc, or the face (the pseudo-normal sign picks its normal by it).
enum : int
{
    kRegionA = 0,
    kRegionB = 1,
    kRegionC = 2,
    kRegionAB = 3,
    kRegionAC = 4,
    kRegionBC = 5,
    kRegionFace = 6
};

// closestPointOnTriangle (KdTree.h:26-74): Ericson's Voronoi-region method;
// *region (may be NULL) receives the region whose branch returned.
__device__ d3 closest_point(const d3& p, const d3& a, const d3& b, const d3& c, int* region = nullptr)
{
    const d3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0)
    {
        if (region) *region = kRegionA;
        return a;
    }
    const d3 bp = sub(p, b);
    const double d3_ = dot(ab, bp), d4 = dot(ac, bp);
    if (d3_ >= 0.0 && d4 <= d3_)
    {
        if (region) *region = kRegionB;
        return b;
    }
    const double vc = d1 * d4 - d3_ * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0)
    {
        if (region) *region = kRegionAB;
        const double v = d1 / (d1 - d3_);
        return mk(a.x + v * ab.x, a.y + v * ab.y, a.z + v * ab.z);
    }
    const d3 cp = sub(p, c);
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6)
    {
        if (region) *region = kRegionC;
        return c;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0)
    {
        if (region) *region = kRegionAC;
        const double w = d2 / (d2 - d6);
        return mk(a.x + w * ac.x, a.y + w * ac.y, a.z + w * ac.z);
    }
    const double va = d3_ * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3_) >= 0.0 && (d5 - d6) >= 0.0)
    {
        if (region) *region = kRegionBC;
        const double w = (d4 - d3_) / ((d4 - d3_) + (d5 - d6));
        return mk(b.x + w * (c.x - b.x), b.y + w * (c.y - b.y), b.z + w * (c.z - b.z));
    }
    if (region) *region = kRegionFace;
    const double denom = 1.0 / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    return mk(a.x + ab.x * v + ac.x * w, a.y + ab.y * v + ac.y * w, a.z + ab.z * v + ac.z * w);
}

// Face normal kept with the nearest triangle (KdTree.h:310-314).
__device__ d3 face_normal(const d3& a, const d3& b, const d3& c)
{
    const d3 n = cross(sub(b, a), sub(c, a));
    const double len = sqrt(dot(n, n));
    if (len > 1.0e-15) return mk(n.x / len, n.y / len, n.z / len);
    return mk(0.0, 0.0, 1.0);
}

// rayIntersectsTriangle (KdTree.h:362-396): Moller-Trumbore, eps 1e-12.
__device__ bool ray_hits(const d3& o, const d3& dir, const d3& a, const d3& b, const d3& c)
{
    const double eps = 1.0e-12;
    const d3 e1 = sub(b, a), e2 = sub(c, a);
    const d3 h = cross(dir, e2);
    const double det = dot(e1, h);
    if (fabs(det) < eps) return false;
    const double invDet = 1.0 / det;
    const d3 s = sub(o, a);
    const double u = invDet * dot(s, h);
    if (u < -eps || u > 1.0 + eps) return false;
    const d3 q = cross(s, e1);
    const double v = invDet * dot(dir, q);
    if (v < -eps || u + v > 1.0 + eps) return false;
    const double t = invDet * dot(e2, q);
    return t > eps;
}

// ---------------------------------------------------------------------------
// LBVH
// ---------------------------------------------------------------------------
struct LbvhView
{
    const float4* nodes;  // 4 float4 per internal node
    const double* tri9;   // leaf order, 9 doubles per triangle
    const int32_t* tri_id; // leaf order -> original triangle index
    int n;                 // triangles
    double dir[3];         // parity ray direction (FP64)
    float inv_dir[3];
    // pseudo-normal sign mode: 18 doubles per slot (vertex a, b, c, edge ab,
    // ac, bc pseudo-normals); NULL: the reference's parity ray
    const double* pn;
    int stackless; // traverse by parent links (no per-thread stack)
};

template <class Tree>
__device__ __forceinline__ d3 tri_vertex(const Tree& b, int slot, int v)
{
    const double* t = b.tri9 + 9 * (int64_t)slot + 3 * v;
    return mk(__ldg(t), __ldg(t + 1), __ldg(t + 2));
}

__device__ __forceinline__ uint64_t spread21(uint64_t x)
{
    x &= 0x1fffffULL;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}

__global__ void k_morton(const double* __restrict__ verts, const int32_t* __restrict__ tris, int n,
                         double3 lo, double3 inv_ext, uint64_t* __restrict__ keys,
                         int32_t* __restrict__ ids)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double c[3] = {0, 0, 0};
    for (int v = 0; v < 3; ++v)
    {
        const int vi = tris[3 * t + v];
        for (int a = 0; a < 3; ++a) c[a] += verts[3 * vi + a];
    }
    const double l[3] = {lo.x, lo.y, lo.z}, ie[3] = {inv_ext.x, inv_ext.y, inv_ext.z};
    uint64_t m = 0;
    for (int a = 0; a < 3; ++a)
    {
        double f = (c[a] / 3.0 - l[a]) * ie[a];
        f = f < 0.0 ? 0.0 : (f > 1.0 ? 1.0 : f);
        const uint64_t q = (uint64_t)(f * 2097151.0);
        m |= spread21(q) << (2 - a);
    }
    keys[t] = m;
    ids[t] = t;
}

__global__ void k_gather_tris(const double* __restrict__ verts, const int32_t* __restrict__ tris,
                              const int32_t* __restrict__ sorted_ids, int n,
                              double* __restrict__ tri9, double* __restrict__ box64)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int t = sorted_ids[s];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v = 0; v < 3; ++v)
    {
        const int vi = tris[3 * t + v];
        for (int a = 0; a < 3; ++a)
        {
            const double x = verts[3 * vi + a];
            tri9[9 * (int64_t)s + 3 * v + a] = x;
            lo[a] = fmin(lo[a], x);
            hi[a] = fmax(hi[a], x);
        }
    }
    // leaves occupy unified indices n-1 .. 2n-2
    double* b = box64 + 6 * (int64_t)(n - 1 + s);
    for (int a = 0; a < 3; ++a)
    {
        b[a] = lo[a];
        b[3 + a] = hi[a];
    }
}

__device__ __forceinline__ int delta(const uint64_t* keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz(i ^ j);
    return __clzll(a ^ b);
}

// Karras 2012, Algorithm 2: one thread per internal node.  Unified node
// indices: internal 0..n-2, leaf s at n-1+s.
__global__ void k_karras(const uint64_t* __restrict__ keys, int n, int2* __restrict__ children,
                         int32_t* __restrict__ parent)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(keys, n, i, j);
    int s = 0;
    int t = l;
    do
    {
        t = (t + 1) / 2;
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + (d < 0 ? d : 0);
    const int left = (min(i, j) == gamma) ? (n - 1 + gamma) : gamma;
    const int right = (max(i, j) == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
    children[i] = make_int2(left, right);
    parent[left] = i;
    parent[right] = i;
}

// Bottom-up box refit: each leaf walks to the root; the second thread to
// arrive at a node unions its children.  No waiting: the first arrival exits.
__global__ void k_refit(int n, const int2* __restrict__ children, const int32_t* __restrict__ parent,
                        int* __restrict__ arrivals, double* box64)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int node = parent[n - 1 + s];
    while (node >= 0)
    {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1) == 0) return;
        __threadfence();
        const int2 c = children[node];
        double lo[3], hi[3];
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = fmin(__ldcg(box64 + 6 * (int64_t)c.x + a), __ldcg(box64 + 6 * (int64_t)c.y + a));
            hi[a] = fmax(__ldcg(box64 + 6 * (int64_t)c.x + 3 + a), __ldcg(box64 + 6 * (int64_t)c.y + 3 + a));
        }
        for (int a = 0; a < 3; ++a)
        {
            __stcg(box64 + 6 * (int64_t)node + a, lo[a]);
            __stcg(box64 + 6 * (int64_t)node + 3 + a, hi[a]);
        }
        node = node == 0 ? -1 : parent[node];
    }
}

// Pack internal nodes: {L.lo, L.hi, R.lo, R.hi} in FP32 rounded outward and
// widened by `margin`; children as node index (internal) or ~slot (leaf).
__global__ void k_pack(int n, const int2* __restrict__ children, const int32_t* __restrict__ parent,
                       const double* __restrict__ box64, double margin, float4* __restrict__ nodes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int2 c = children[i];
    float f[12];
    const int ch[2] = {c.x, c.y};
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a)
        {
            f[6 * k + a] = __double2float_rd(box64[6 * (int64_t)ch[k] + a] - margin);
            f[6 * k + 3 + a] = __double2float_ru(box64[6 * (int64_t)ch[k] + 3 + a] + margin);
        }
    const int enc[2] = {c.x >= n - 1 ? ~(c.x - (n - 1)) : c.x, c.y >= n - 1 ? ~(c.y - (n - 1)) : c.y};
    float4* o = nodes + 4 * (int64_t)i;
    o[0] = make_float4(f[0], f[1], f[2], f[3]);
    o[1] = make_float4(f[4], f[5], f[6], f[7]);
    o[2] = make_float4(f[8], f[9], f[10], f[11]);
    // children (leaves as ~slot) and the parent (-1 at the root), for the
    // stackless traversals
    o[3] = make_float4(__int_as_float(enc[0]), __int_as_float(enc[1]), __int_as_float(parent[i]), 0.f);
}

// ---------------------------------------------------------------------------
// traversal
// ---------------------------------------------------------------------------
__device__ __forceinline__ float box_dist2(const float p[3], float lx, float ly, float lz, float hx,
                                           float hy, float hz)
{
    const float dx = fmaxf(fmaxf(lx - p[0], p[0] - hx), 0.f);
    const float dy = fmaxf(fmaxf(ly - p[1], p[1] - hy), 0.f);
    const float dz = fmaxf(fmaxf(lz - p[2], p[2] - hz), 0.f);
    return dx * dx + dy * dy + dz * dz;
}

struct Nearest
{
    double sq;
    int slot;
    int id;
    d3 cp;
    int region; // Voronoi region of cp on the triangle
};

__device__ __forceinline__ void test_triangle(const LbvhView& b, const d3& p, int slot, Nearest& best)
{
    const d3 a = tri_vertex(b, slot, 0), bb = tri_vertex(b, slot, 1), c = tri_vertex(b, slot, 2);
    int region;
    const d3 cp = closest_point(p, a, bb, c, &region);
    const d3 d = sub(p, cp);
    const double sq = dot(d, d);
    const int id = __ldg(b.tri_id + slot);
    if (sq < best.sq || (sq == best.sq && id < best.id))
    {
        best.sq = sq;
        best.slot = slot;
        best.id = id;
        best.cp = cp;
        best.region = region;
    }
}

// Traversal work of one query, counted only by the instrumented (COUNT)
// instantiations of the traversals below: nodes whose children (or
// triangles) were examined and triangles tested, for the nearest search and
// for the parity ray.
struct TravCount
{
    int nearest_nodes = 0, nearest_tris = 0, ray_nodes = 0, ray_tris = 0;
    int nearest_exact = 0; // closest-point tests left after the box cull
};

// Upper bound used for FP32 culling: bestSq rounded up, plus a relative slack
// covering FP32 rounding of the box distance.
__device__ __forceinline__ float cull_limit(double sq)
{
    return sq >= 3.0e38 ? INFINITY : __double2float_ru(sq) * 1.000002f;
}

// The stackless form of the LBVH nearest search: the same near-first order
// and the same pruning decisions as the stack form below, taken at the same
// moments, by walking parent links.  At a node the walk knows where it came
// from: from the parent (try the near child, else the far one), from the
// near child (try the far one) or from the far child (go up); a child is
// entered when its box distance is within the cull limit of the current
// best, which is when the stack form pushes or pops it.  Leaf children are
// tested in place.  Returns the same triangle (the lowest id at equal
// distance does not depend on the order) and counts the same work.
template <bool COUNT>
__device__ void nearest_stackless(const LbvhView& b, const d3& p, const float pf[3], Nearest& best,
                                  TravCount* tc)
{
    enum : int
    {
        kFromParent = 0,
        kFromNear = 1,
        kFromFar = 2,
        kFromChild = 3
    };
    int node = 0, state = kFromParent, child = -1;
    while (true)
    {
        if constexpr (COUNT)
            if (state == kFromParent) ++tc->nearest_nodes;
        const float4 n0 = __ldg(b.nodes + 4 * (int64_t)node);
        const float4 n1 = __ldg(b.nodes + 4 * (int64_t)node + 1);
        const float4 n2 = __ldg(b.nodes + 4 * (int64_t)node + 2);
        const float4 n3 = __ldg(b.nodes + 4 * (int64_t)node + 3);
        const float dl = box_dist2(pf, n0.x, n0.y, n0.z, n0.w, n1.x, n1.y);
        const float dr = box_dist2(pf, n1.z, n1.w, n2.x, n2.y, n2.z, n2.w);
        const int cl = __float_as_int(n3.x), cr = __float_as_int(n3.y);
        const bool lfirst = dl <= dr;
        const int nearc = lfirst ? cl : cr, farc = lfirst ? cr : cl;
        const float dn = lfirst ? dl : dr, df = lfirst ? dr : dl;
        if (state == kFromChild) state = child == nearc ? kFromNear : kFromFar;
        const float lim = cull_limit(best.sq);
        int next = 0;
        bool go = false;
        if (state == kFromParent && dn <= lim)
        {
            next = nearc;
            go = true;
        }
        else if (state != kFromFar && df <= lim)
        {
            next = farc;
            go = true;
        }
        if (go)
        {
            const bool is_near = state == kFromParent && next == nearc;
            if (next < 0)
            {
                if constexpr (COUNT) ++tc->nearest_tris;
                test_triangle(b, p, ~next, best);
                state = is_near ? kFromNear : kFromFar;
                continue;
            }
            node = next;
            state = kFromParent;
            continue;
        }
        const int parent = __float_as_int(n3.z);
        if (parent < 0) break;
        child = node;
        node = parent;
        state = kFromChild;
    }
}

// init_sq: a triangle is recorded only below it (default +inf).
template <bool COUNT = false>
__device__ Nearest tree_nearest(const LbvhView& b, const d3& p, int* status, TravCount* tc = nullptr,
                                double init_sq = 1.0e308 * 10.0)
{
    Nearest best;
    best.sq = init_sq;
    best.slot = -1;
    best.id = 0x7fffffff;
    best.cp = p;
    best.region = kRegionFace;
    if (b.n == 1)
    {
        if constexpr (COUNT) ++tc->nearest_tris;
        test_triangle(b, p, 0, best);
        return best;
    }
    if (b.stackless)
    {
        const float pf[3] = {(float)p.x, (float)p.y, (float)p.z};
        nearest_stackless<COUNT>(b, p, pf, best, tc);
        return best;
    }
    const float pf[3] = {(float)p.x, (float)p.y, (float)p.z};
    int stack[kStackDepth];
    float sdist[kStackDepth];
    int sp = 0;
    int node = 0;
    while (true)
    {
        if (node < 0)
        {
            if constexpr (COUNT) ++tc->nearest_tris;
            test_triangle(b, p, ~node, best);
        }
        else
        {
            if constexpr (COUNT) ++tc->nearest_nodes;
            const float4 n0 = __ldg(b.nodes + 4 * (int64_t)node);
            const float4 n1 = __ldg(b.nodes + 4 * (int64_t)node + 1);
            const float4 n2 = __ldg(b.nodes + 4 * (int64_t)node + 2);
            const float4 n3 = __ldg(b.nodes + 4 * (int64_t)node + 3);
            const float dl = box_dist2(pf, n0.x, n0.y, n0.z, n0.w, n1.x, n1.y);
            const float dr = box_dist2(pf, n1.z, n1.w, n2.x, n2.y, n2.z, n2.w);
            const int cl = __float_as_int(n3.x), cr = __float_as_int(n3.y);
            const float lim = cull_limit(best.sq);
            const bool hl = dl <= lim, hr = dr <= lim;
            if (hl && hr)
            {
                const bool lfirst = dl <= dr;
                if (sp < kStackDepth)
                {
                    stack[sp] = lfirst ? cr : cl;
                    sdist[sp] = lfirst ? dr : dl;
                    ++sp;
                }
                else
                {
                    atomicOr(status, kStatusStackOverflow);
                }
                node = lfirst ? cl : cr;
                continue;
            }
            if (hl)
            {
                node = cl;
                continue;
            }
            if (hr)
            {
                node = cr;
                continue;
            }
        }
        // pop the next subtree that can still hold a closer triangle
        bool found = false;
        while (sp > 0)
        {
            --sp;
            if (sdist[sp] <= cull_limit(best.sq))
            {
                node = stack[sp];
                found = true;
                break;
            }
        }
        if (!found) break;
    }
    return best;
}

__device__ __forceinline__ bool ray_box(const float o[3], const float inv[3], float lx, float ly,
                                        float lz, float hx, float hy, float hz)
{
    float t0 = (lx - o[0]) * inv[0], t1 = (hx - o[0]) * inv[0];
    float tmin = fminf(t0, t1), tmax = fmaxf(t0, t1);
    t0 = (ly - o[1]) * inv[1];
    t1 = (hy - o[1]) * inv[1];
    tmin = fmaxf(tmin, fminf(t0, t1));
    tmax = fminf(tmax, fmaxf(t0, t1));
    t0 = (lz - o[2]) * inv[2];
    t1 = (hz - o[2]) * inv[2];
    tmin = fmaxf(tmin, fminf(t0, t1));
    tmax = fminf(tmax, fmaxf(t0, t1));
    tmin = fmaxf(tmin, 0.f);
    return tmax >= tmin;
}

// The parity ray's count by parent links (left child first; the count does
// not depend on the order): from the parent try the left child, else the
// right; from the left child try the right; from the right go up.
template <bool COUNT>
__device__ int ray_count_stackless(const LbvhView& b, const d3& p, const d3& dir, const float o[3], TravCount* tc)
{
    int node = 0, state = 0, child = -1, hits = 0; // state: 0 from parent, 1 from left, 2 from right, 3 from a child
    while (true)
    {
        if constexpr (COUNT)
            if (state == 0) ++tc->ray_nodes;
        const float4 n0 = __ldg(b.nodes + 4 * (int64_t)node);
        const float4 n1 = __ldg(b.nodes + 4 * (int64_t)node + 1);
        const float4 n2 = __ldg(b.nodes + 4 * (int64_t)node + 2);
        const float4 n3 = __ldg(b.nodes + 4 * (int64_t)node + 3);
        const int cl = __float_as_int(n3.x), cr = __float_as_int(n3.y);
        if (state == 3) state = child == cl ? 1 : 2;
        int next = 0;
        bool go = false;
        if (state == 0 && ray_box(o, b.inv_dir, n0.x, n0.y, n0.z, n0.w, n1.x, n1.y))
        {
            next = cl;
            go = true;
        }
        else if (state != 2 && ray_box(o, b.inv_dir, n1.z, n1.w, n2.x, n2.y, n2.z, n2.w))
        {
            next = cr;
            go = true;
        }
        if (go)
        {
            const bool left = state == 0 && next == cl;
            if (next < 0)
            {
                if constexpr (COUNT) ++tc->ray_tris;
                const int s = ~next;
                hits += ray_hits(p, dir, tri_vertex(b, s, 0), tri_vertex(b, s, 1), tri_vertex(b, s, 2)) ? 1 : 0;
                state = left ? 1 : 2;
                continue;
            }
            node = next;
            state = 0;
            continue;
        }
        const int parent = __float_as_int(n3.z);
        if (parent < 0) break;
        child = node;
        node = parent;
        state = 3;
    }
    return hits;
}

// countRayIntersections (KdTree.h:398-441): number of triangles the fixed
// ray hits (exact FP64 test on every triangle whose widened box it crosses).
template <bool COUNT = false>
__device__ int tree_ray_count(const LbvhView& b, const d3& p, int* status, TravCount* tc = nullptr)
{
    const d3 dir = mk(b.dir[0], b.dir[1], b.dir[2]);
    if (b.n == 1)
    {
        if constexpr (COUNT) ++tc->ray_tris;
        return ray_hits(p, dir, tri_vertex(b, 0, 0), tri_vertex(b, 0, 1), tri_vertex(b, 0, 2)) ? 1 : 0;
    }
    const float o[3] = {(float)p.x, (float)p.y, (float)p.z};
    if (b.stackless) return ray_count_stackless<COUNT>(b, p, dir, o, tc);
    int stack[kStackDepth];
    int sp = 0;
    int node = 0;
    int hits = 0;
    while (true)
    {
        if (node < 0)
        {
            if constexpr (COUNT) ++tc->ray_tris;
            const int s = ~node;
            hits += ray_hits(p, dir, tri_vertex(b, s, 0), tri_vertex(b, s, 1), tri_vertex(b, s, 2)) ? 1 : 0;
        }
        else
        {
            if constexpr (COUNT) ++tc->ray_nodes;
            const float4 n0 = __ldg(b.nodes + 4 * (int64_t)node);
            const float4 n1 = __ldg(b.nodes + 4 * (int64_t)node + 1);
            const float4 n2 = __ldg(b.nodes + 4 * (int64_t)node + 2);
            const float4 n3 = __ldg(b.nodes + 4 * (int64_t)node + 3);
            const bool hl = ray_box(o, b.inv_dir, n0.x, n0.y, n0.z, n0.w, n1.x, n1.y);
            const bool hr = ray_box(o, b.inv_dir, n1.z, n1.w, n2.x, n2.y, n2.z, n2.w);
            const int cl = __float_as_int(n3.x), cr = __float_as_int(n3.y);
            if (hl && hr)
            {
                if (sp < kStackDepth)
                    stack[sp++] = cr;
                else
                    atomicOr(status, kStatusStackOverflow);
                node = cl;
                continue;
            }
            if (hl)
            {
                node = cl;
                continue;
            }
            if (hr)
            {
                node = cr;
                continue;
            }
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return hits;
}

// ---------------------------------------------------------------------------
// reference-order tree: the reference's median-split BVH, traversed on the
// device in the reference's order with FP64 boxes
// ---------------------------------------------------------------------------
struct RefNode
{
    double lo[3];
    double hi[3];
    int left, right; // internal: children (node ids)
    int start, count; // leaf: range of slots (count > 0)
};
static_assert(sizeof(RefNode) == 64, "RefNode is one 64-byte record");

struct RefTreeView
{
    const RefNode* nodes;
    const double* tri9;    // slot order (m_indices), 9 doubles per triangle
    const int32_t* tri_id; // slot -> original triangle index
    int n;
    int nnodes;
    double dir[3];
    // Per-triangle FP32 boxes for the cull ahead of the FP64 closest-point
    // test (2 float4 per slot: lo, hi; NULL: no cull) and its margins, set
    // from the scene extent E: cull_m = 2^-21 E (rounded up), cull_abs =
    // (2^-20 E)^2.
    const float4* tbox;
    float cull_m;
    double cull_abs;
    const double* pn; // pseudo-normals per slot as in LbvhView (NULL: parity ray)
};

// Cull margins of a scene whose points and vertices lie within |x| <= E.
inline void set_cull_margins(RefTreeView& v, double extent)
{
    v.cull_m = (float)std::ldexp(extent, -20); // >= 2^-21 E after rounding
    const double a = std::ldexp(extent, -20);
    v.cull_abs = a * a;
}

// Conservative FP32 box of each triangle in slot order (lo rounded down, hi
// rounded up, so it contains the FP64 triangle).  A near-degenerate triangle
// -- |ab x ac|^2 <= 2^-20 (longest edge)^4, where the closest point's
// barycentric division is ill-conditioned -- gets an unbounded box and is
// never culled.
__global__ void k_tri_boxes(const double* __restrict__ tri9, int n, float4* __restrict__ tbox)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double* t = tri9 + 9 * (int64_t)s;
    const d3 a = mk(t[0], t[1], t[2]), b = mk(t[3], t[4], t[5]), c = mk(t[6], t[7], t[8]);
    const d3 ab = sub(b, a), ac = sub(c, a), bc = sub(c, b);
    const d3 cr = cross(ab, ac);
    const double e2 = fmax(dot(ab, ab), fmax(dot(ac, ac), dot(bc, bc)));
    const bool degenerate = !(dot(cr, cr) > 0x1p-20 * e2 * e2);
    float4 lo, hi;
    if (degenerate)
    {
        lo = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
        hi = make_float4(INFINITY, INFINITY, INFINITY, 0.f);
    }
    else
    {
        lo = make_float4(__double2float_rd(fmin(a.x, fmin(b.x, c.x))), __double2float_rd(fmin(a.y, fmin(b.y, c.y))),
                         __double2float_rd(fmin(a.z, fmin(b.z, c.z))), 0.f);
        hi = make_float4(__double2float_ru(fmax(a.x, fmax(b.x, c.x))), __double2float_ru(fmax(a.y, fmax(b.y, c.y))),
                         __double2float_ru(fmax(a.z, fmax(b.z, c.z))), 0.f);
    }
    tbox[2 * (int64_t)s] = lo;
    tbox[2 * (int64_t)s + 1] = hi;
}

// The cull bound for a best squared distance `sq`: a triangle whose FP32 box
// lower bound exceeds it cannot produce a computed squared distance below
// `sq` (the reference's strict update), by the margins above: FP32 rounding
// of the point and the box gap (< 2^-21 E per axis, taken off each gap),
// FP32 rounding of the squares and sum (the factor 1 - 2^-19), and the
// rounding of the FP64 closest point of a well-conditioned triangle
// (covered by 2^-16 relative and (2^-20 E)^2 absolute on `sq`).
__device__ __forceinline__ float cull_bound(const RefTreeView& b, double sq)
{
    return __double2float_ru(sq * (1.0 + 0x1p-16) + b.cull_abs);
}

__device__ __forceinline__ bool box_culled(const RefTreeView& b, int s, const float pf[3], float bound)
{
    const float4 lo = __ldg(b.tbox + 2 * (int64_t)s), hi = __ldg(b.tbox + 2 * (int64_t)s + 1);
    const float gx = fmaxf(fmaxf(fmaxf(lo.x - pf[0], pf[0] - hi.x), 0.f) - b.cull_m, 0.f);
    const float gy = fmaxf(fmaxf(fmaxf(lo.y - pf[1], pf[1] - hi.y), 0.f) - b.cull_m, 0.f);
    const float gz = fmaxf(fmaxf(fmaxf(lo.z - pf[2], pf[2] - hi.z), 0.f) - b.cull_m, 0.f);
    const float sum = gx * gx + gy * gy + gz * gz;
    return sum * (1.f - 0x1p-19f) > bound;
}

__device__ __forceinline__ void load_box(const RefNode* nd, double lo[3], double hi[3])
{
    const double2* q = reinterpret_cast<const double2*>(nd);
    const double2 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    lo[0] = a.x;
    lo[1] = a.y;
    lo[2] = b.x;
    hi[0] = b.y;
    hi[1] = c.x;
    hi[2] = c.y;
}

// squaredDistanceToAabb (KdTree.h:244-264), same branches and order.
__device__ __forceinline__ double box_dist_sq(const d3& p, const double lo[3], const double hi[3])
{
    const double pp[3] = {p.x, p.y, p.z};
    double sq = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        if (pp[a] < lo[a])
        {
            const double d = lo[a] - pp[a];
            sq += d * d;
        }
        else if (pp[a] > hi[a])
        {
            const double d = pp[a] - hi[a];
            sq += d * d;
        }
    }
    return sq;
}

// searchNearest (KdTree.h:266-328) without recursion: the explicit stack pops
// subtrees in the same near-first depth-first order and applies the same
// "box distance > best" cut when a subtree is entered, and triangles replace
// the best only on a strictly smaller squared distance -- so the triangle
// found is the reference's, ties included.
// init_sq: a triangle is recorded only below it (default: the reference's
// DBL_MAX start).
template <bool COUNT = false>
__device__ Nearest tree_nearest(const RefTreeView& b, const d3& p, int* status, TravCount* tc = nullptr,
                                double init_sq = DBL_MAX)
{
    Nearest best;
    best.sq = init_sq;
    best.slot = -1;
    best.id = -1;
    best.cp = mk(0.0, 0.0, 0.0);
    best.region = kRegionFace;
    if (b.nnodes == 0) return best;
    const float pf[3] = {(float)p.x, (float)p.y, (float)p.z};
    float bound = cull_bound(b, init_sq);
    int stack[kStackDepth];
    double sdist[kStackDepth];
    int sp = 0;
    {
        double lo[3], hi[3];
        load_box(b.nodes, lo, hi);
        stack[0] = 0;
        sdist[0] = box_dist_sq(p, lo, hi);
        sp = 1;
    }
    while (sp > 0)
    {
        --sp;
        const int node = stack[sp];
        if (sdist[sp] > best.sq) continue;
        if constexpr (COUNT) ++tc->nearest_nodes;
        const RefNode* nd = b.nodes + node;
        const int4 meta = __ldg(reinterpret_cast<const int4*>(nd) + 3);
        if (meta.w > 0)
        {
            if constexpr (COUNT) tc->nearest_tris += meta.w;
            for (int s = meta.z; s < meta.z + meta.w; ++s)
            {
                // exact-decision cull: a triangle skipped here could not
                // have replaced the best (see cull_bound)
                if (b.tbox && box_culled(b, s, pf, bound)) continue;
                if constexpr (COUNT) ++tc->nearest_exact;
                const d3 a = tri_vertex(b, s, 0), bb = tri_vertex(b, s, 1), c = tri_vertex(b, s, 2);
                int region;
                const d3 cp = closest_point(p, a, bb, c, &region);
                const d3 d = sub(p, cp);
                const double sq = dot(d, d);
                if (sq < best.sq)
                {
                    best.sq = sq;
                    best.slot = s;
                    best.cp = cp;
                    best.region = region;
                    bound = cull_bound(b, sq);
                }
            }
            continue;
        }
        double llo[3], lhi[3], rlo[3], rhi[3];
        load_box(b.nodes + meta.x, llo, lhi);
        load_box(b.nodes + meta.y, rlo, rhi);
        const double dl = box_dist_sq(p, llo, lhi);
        const double dr = box_dist_sq(p, rlo, rhi);
        int first = meta.x, second = meta.y;
        double df = dl, ds = dr;
        if (dr < dl)
        {
            first = meta.y;
            second = meta.x;
            df = dr;
            ds = dl;
        }
        if (sp + 2 > kStackDepth)
        {
            atomicOr(status, kStatusStackOverflow);
            break;
        }
        stack[sp] = second;
        sdist[sp] = ds;
        ++sp;
        stack[sp] = first;
        sdist[sp] = df;
        ++sp;
    }
    if (best.slot >= 0) best.id = __ldg(b.tri_id + best.slot);
    return best;
}

// rayIntersectsAabb (KdTree.h:335-360), same arithmetic.
__device__ __forceinline__ bool ray_box_ref(const d3& o, const double dir[3], const double lo[3],
                                            const double hi[3])
{
    const double oo[3] = {o.x, o.y, o.z};
    double tmin = 0.0, tmax = DBL_MAX;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        const double invD = 1.0 / dir[a];
        double t0 = (lo[a] - oo[a]) * invD;
        double t1 = (hi[a] - oo[a]) * invD;
        if (t0 > t1)
        {
            const double t = t0;
            t0 = t1;
            t1 = t;
        }
        tmin = tmin < t0 ? t0 : tmin;
        tmax = t1 < tmax ? t1 : tmax;
        if (tmax < tmin) return false;
    }
    return true;
}

// countRayIntersectionsRecursive (KdTree.h:398-441) over the same tree.
template <bool COUNT = false>
__device__ int tree_ray_count(const RefTreeView& b, const d3& p, int* status, TravCount* tc = nullptr)
{
    if (b.nnodes == 0) return 0;
    const d3 dir = mk(b.dir[0], b.dir[1], b.dir[2]);
    int stack[kStackDepth];
    int sp = 0;
    stack[sp++] = 0;
    int hits = 0;
    while (sp > 0)
    {
        const int node = stack[--sp];
        const RefNode* nd = b.nodes + node;
        double lo[3], hi[3];
        load_box(nd, lo, hi);
        if constexpr (COUNT) ++tc->ray_nodes;
        if (!ray_box_ref(p, b.dir, lo, hi)) continue;
        const int4 meta = __ldg(reinterpret_cast<const int4*>(nd) + 3);
        if (meta.w > 0)
        {
            if constexpr (COUNT) tc->ray_tris += meta.w;
            for (int s = meta.z; s < meta.z + meta.w; ++s)
                hits += ray_hits(p, dir, tri_vertex(b, s, 0), tri_vertex(b, s, 1), tri_vertex(b, s, 2)) ? 1 : 0;
            continue;
        }
        if (sp + 2 > kStackDepth)
        {
            atomicOr(status, kStatusStackOverflow);
            break;
        }
        stack[sp++] = meta.y;
        stack[sp++] = meta.x;
    }
    return hits;
}

struct SignedResult
{
    double sd;
    d3 cp;
    d3 fn;
};

// findSignedNearest (KdTree.h:143-165).
template <class Tree, bool COUNT = false>
__device__ SignedResult signed_nearest(const Tree& b, const d3& p, int* status, TravCount* tc = nullptr)
{
    const Nearest best = tree_nearest<COUNT>(b, p, status, tc);
    SignedResult r;
    const double dist = sqrt(best.sq);
    r.cp = best.cp;
    r.fn = best.slot >= 0 ? face_normal(tri_vertex(b, best.slot, 0), tri_vertex(b, best.slot, 1),
                                        tri_vertex(b, best.slot, 2))
                          : mk(0.0, 0.0, 1.0);
    if (b.pn && best.slot >= 0)
    {
        // pseudo-normal sign: the normal of the closest point's feature --
        // the face normal in the face, else the angle-weighted vertex or the
        // edge pseudo-normal, which every triangle sharing that vertex or
        // edge carries alike, so the sign does not depend on which of the
        // equidistant triangles the search kept
        d3 n = r.fn;
        if (best.region < kRegionFace)
        {
            const double* q = b.pn + 18 * (int64_t)best.slot + 3 * best.region;
            n = mk(__ldg(q), __ldg(q + 1), __ldg(q + 2));
        }
        r.sd = dot(sub(p, r.cp), n) >= 0.0 ? dist : -dist;
        return r;
    }
    const int hits = tree_ray_count<COUNT>(b, p, status, tc);
    if (hits > 0)
        r.sd = (hits % 2) == 1 ? -dist : dist;
    else
        r.sd = dot(sub(p, r.cp), r.fn) >= 0.0 ? dist : -dist;
    return r;
}

// SdfBuilder.cpp:1070-1085 normal: sign * (c - cp) / |c - cp|, or the signed
// face normal within 1e-12 of the surface.
__device__ __forceinline__ d3 voxel_normal(const d3& c, const SignedResult& r)
{
    const d3 diff = sub(c, r.cp);
    const double dist = sqrt(dot(diff, diff));
    const double sign = r.sd >= 0.0 ? 1.0 : -1.0;
    if (dist > 1e-12) return mk(sign * diff.x / dist, sign * diff.y / dist, sign * diff.z / dist);
    return mk(sign * r.fn.x, sign * r.fn.y, sign * r.fn.z);
}

struct SpecD
{
    double bmin[3];
    double voxel[3];
    int n[3];
};

__device__ __forceinline__ d3 voxel_center(const SpecD& s, int i, int j, int k)
{
    // GridSpec::centerFromIndex (GridSpec.h:29-33)
    return mk(s.bmin[0] + s.voxel[0] * (i + 0.5), s.bmin[1] + s.voxel[1] * (j + 0.5),
              s.bmin[2] + s.voxel[2] * (k + 0.5));
}

// Resident CTAs per SM the fill kernels ask the register allocator for: 3
// (at most 80 registers, a few words of spills) against the 85-99 registers
// and 2 CTAs the allocator picks unasked measured 7% faster on the 512^3
// icosphere's sparse fill (82.2 -> 76.1 ms) and 4% on the hollow cylinder's
// dense fill, with identical results.
#ifndef SDFO_FILL_MIN_BLOCKS
#define SDFO_FILL_MIN_BLOCKS 3
#endif

// Voxel tile of a 256-thread fill CTA: 2^lx x 2^ly x 256 / 2^(lx+ly) voxels,
// x fastest, so a warp covers a 2^lx x min(2^ly, 32 / 2^lx) x .. patch
// (default 8 x 8 x 4: warps of 8 x 4 x 1; 4 x 4 x 16: warps of 4 x 4 x 2).
struct FillTile
{
    int lx, ly;
    __host__ __device__ int x() const { return 1 << lx; }
    __host__ __device__ int y() const { return 1 << ly; }
    __host__ __device__ int z() const { return 256 >> (lx + ly); }
    dim3 grid(const SpecD& s) const
    {
        return dim3((s.n[0] + x() - 1) / x(), (s.n[1] + y() - 1) / y(), (s.n[2] + z() - 1) / z());
    }
    __device__ void voxel(int& i, int& j, int& k) const
    {
        const int tx = threadIdx.x;
        i = blockIdx.x * x() + (tx & (x() - 1));
        j = blockIdx.y * y() + ((tx >> lx) & (y() - 1));
        k = blockIdx.z * z() + (tx >> (lx + ly));
    }
};

// Dense fill: CTA = one voxel tile (coherent traversals), thread = voxel.
template <class Tree>
__global__ void __launch_bounds__(256, SDFO_FILL_MIN_BLOCKS) k_dense_fill(Tree b, SpecD s, FillTile t,
                                                    double* __restrict__ phi64,
                                                    double* __restrict__ n64, double* __restrict__ w64,
                                                    float4* __restrict__ phin, int* status)
{
    int i, j, k;
    t.voxel(i, j, k);
    if (i >= s.n[0] || j >= s.n[1] || k >= s.n[2]) return;
    const int64_t idx = i + (int64_t)s.n[0] * (j + (int64_t)s.n[1] * k);
    const d3 c = voxel_center(s, i, j, k);
    const SignedResult r = signed_nearest(b, c, status);
    const d3 g = voxel_normal(c, r);
    phi64[idx] = r.sd;
    n64[3 * idx + 0] = g.x;
    n64[3 * idx + 1] = g.y;
    n64[3 * idx + 2] = g.z;
    if (w64)
    {
        w64[3 * idx + 0] = r.cp.x;
        w64[3 * idx + 1] = r.cp.y;
        w64[3 * idx + 2] = r.cp.z;
    }
    phin[idx] = make_float4((float)r.sd, (float)g.x, (float)g.y, (float)g.z);
}

// The dense fill's traversals over the same voxels and tiles, counted
// (TravCount) and summed into out[4] instead of stored.
template <class Tree>
__global__ void __launch_bounds__(256) k_dense_count(Tree b, SpecD s, FillTile t, unsigned long long* out,
                                                     int* status)
{
    const int tx = threadIdx.x;
    int i, j, k;
    t.voxel(i, j, k);
    TravCount tc;
    if (i < s.n[0] && j < s.n[1] && k < s.n[2])
        (void)signed_nearest<Tree, true>(b, voxel_center(s, i, j, k), status, &tc);
    unsigned long long v[5] = {(unsigned long long)tc.nearest_nodes, (unsigned long long)tc.nearest_tris,
                               (unsigned long long)tc.ray_nodes, (unsigned long long)tc.ray_tris,
                               (unsigned long long)tc.nearest_exact};
#pragma unroll
    for (int q = 0; q < 5; ++q)
    {
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        if ((tx & 31) == 0) atomicAdd(out + q, v[q]);
    }
}

// Symmetrised central-difference Hessian of the normal field
// (SdfBuilder.cpp:1105-1152): H[:,a] = (n(+a) - n(-a)) / (2 h_a), clamped at
// the boundary, H = (H + H^T) / 2; stored xx, xy, xz, yy, yz, zz.
__device__ __forceinline__ void sym_hessian(const double dn[3][3], double h6[6])
{
    h6[0] = 0.5 * (dn[0][0] + dn[0][0]);
    h6[1] = 0.5 * (dn[1][0] + dn[0][1]);
    h6[2] = 0.5 * (dn[2][0] + dn[0][2]);
    h6[3] = 0.5 * (dn[1][1] + dn[1][1]);
    h6[4] = 0.5 * (dn[2][1] + dn[1][2]);
    h6[5] = 0.5 * (dn[2][2] + dn[2][2]);
}

__global__ void k_dense_hessian(SpecD s, const double* __restrict__ n64, double* __restrict__ h64,
                                float* __restrict__ hess6)
{
    const int64_t total = (int64_t)s.n[0] * s.n[1] * s.n[2];
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int nx = s.n[0], ny = s.n[1], nz = s.n[2];
    const int i = (int)(idx % nx), j = (int)((idx / nx) % ny), k = (int)(idx / ((int64_t)nx * ny));
    const int ip = min(i + 1, nx - 1), im = max(i - 1, 0);
    const int jp = min(j + 1, ny - 1), jm = max(j - 1, 0);
    const int kp = min(k + 1, nz - 1), km = max(k - 1, 0);
    const int64_t pi[3] = {ip + (int64_t)nx * (j + (int64_t)ny * k), i + (int64_t)nx * (jp + (int64_t)ny * k),
                           i + (int64_t)nx * (j + (int64_t)ny * kp)};
    const int64_t mi[3] = {im + (int64_t)nx * (j + (int64_t)ny * k), i + (int64_t)nx * (jm + (int64_t)ny * k),
                           i + (int64_t)nx * (j + (int64_t)ny * km)};
    double dn[3][3];
    for (int a = 0; a < 3; ++a)
        for (int r = 0; r < 3; ++r)
            dn[a][r] = (__ldg(n64 + 3 * pi[a] + r) - __ldg(n64 + 3 * mi[a] + r)) / (2.0 * s.voxel[a]);
    double h6[6];
    sym_hessian(dn, h6);
    for (int q = 0; q < 6; ++q)
    {
        h64[6 * idx + q] = h6[q];
        hess6[6 * idx + q] = (float)h6[q];
    }
}

// Sparse block activation (SdfBuilder.cpp:869-890): distance from the block's
// geometric centre to the mesh against band + halo*h + (sqrt(3)/2)*bd*h.
//
// Most candidate blocks lie far from the surface, where the reference's
// nearest search visits many nodes.  A first search starts with the best
// squared distance set to activation^2 (1 + 1e-9), so it prunes everything
// farther.  If it records no triangle, every triangle's computed squared
// distance is above activation^2: the tested ones by that test, and those
// in pruned subtrees because they lie no nearer than their box, whose
// distance was above the start value.  The reference's search would then
// also return a distance above the activation distance, with a margin far
// beyond FP64 rounding, and the block is inactive.  Otherwise the block
// runs the reference's full search, and its result decides.
template <class Tree>
__device__ __forceinline__ int32_t block_active(const Tree& b, const SpecD& s, int bd, int nbx,
                                                int nby, int bl, double activation, int* status)
{
    const int bi = bl % nbx, bj = (bl / nbx) % nby, bk = bl / (nbx * nby);
    const int i0 = bi * bd, j0 = bj * bd, k0 = bk * bd;
    const int i1 = min(i0 + bd, s.n[0]), j1 = min(j0 + bd, s.n[1]), k1 = min(k0 + bd, s.n[2]);
    const d3 c = mk(s.bmin[0] + s.voxel[0] * (0.5 * (double)(i0 + i1)),
                    s.bmin[1] + s.voxel[1] * (0.5 * (double)(j0 + j1)),
                    s.bmin[2] + s.voxel[2] * (0.5 * (double)(k0 + k1)));
    const Nearest near = tree_nearest(b, c, status, nullptr, activation * activation * (1.0 + 1e-9));
    if (near.slot < 0) return 0;
    const Nearest best = tree_nearest(b, c, status);
    const double dist = sqrt(best.sq);
    return fabs(dist) <= activation ? 1 : 0;
}

template <class Tree>
__global__ void k_sparse_activate(Tree b, SpecD s, int bd, int nbx, int nby, int nbz,
                                  double activation, int32_t* __restrict__ flags, int* status)
{
    const int bl = blockIdx.x * blockDim.x + threadIdx.x;
    if (bl >= nbx * nby * nbz) return;
    flags[bl] = block_active(b, s, bd, nbx, nby, bl, activation, status);
}

__global__ void k_sparse_table(int total, int nbx, int nby, const int32_t* __restrict__ flags,
                               const int32_t* __restrict__ slots, int32_t* __restrict__ table,
                               int32_t* __restrict__ ijk)
{
    const int bl = blockIdx.x * blockDim.x + threadIdx.x;
    if (bl >= total) return;
    if (flags[bl])
    {
        const int slot = slots[bl];
        table[bl] = slot;
        ijk[3 * slot + 0] = bl % nbx;
        ijk[3 * slot + 1] = (bl / nbx) % nby;
        ijk[3 * slot + 2] = bl / (nbx * nby);
    }
    else
    {
        table[bl] = -1;
    }
}

// One voxel of a stored brick (SdfBuilder.cpp:925-965); voxels outside the
// grid get phi 0, n (1,0,0).
template <class Tree>
__device__ __forceinline__ float4 brick_voxel(const Tree& b, const SpecD& s, int bd, int bi,
                                              int bj, int bk, int local, int* status)
{
    const int lx = local % bd, ly = (local / bd) % bd, lz = local / (bd * bd);
    const int i = bi * bd + lx, j = bj * bd + ly, k = bk * bd + lz;
    if (i >= s.n[0] || j >= s.n[1] || k >= s.n[2]) return make_float4(0.f, 1.f, 0.f, 0.f);
    const d3 c = voxel_center(s, i, j, k);
    const SignedResult r = signed_nearest(b, c, status);
    const d3 g = voxel_normal(c, r);
    return make_float4((float)r.sd, (float)g.x, (float)g.y, (float)g.z);
}

// Brick fill: one CTA per stored block.
template <class Tree>
__global__ void __launch_bounds__(256, SDFO_FILL_MIN_BLOCKS) k_sparse_fill(Tree b, SpecD s, int bd,
                                                     const int32_t* __restrict__ ijk,
                                                     float4* __restrict__ phin, int* status)
{
    const int blk = blockIdx.x;
    const int V = bd * bd * bd;
    const int bi = ijk[3 * blk], bj = ijk[3 * blk + 1], bk = ijk[3 * blk + 2];
    for (int local = threadIdx.x; local < V; local += blockDim.x)
        phin[(int64_t)blk * V + local] = brick_voxel(b, s, bd, bi, bj, bk, local, status);
}

// estimateSparseHessian (SdfBuilder.cpp:1154-1225) for stored voxel `local`
// of brick `blk` of one grid: neighbours through the block table, a missing
// neighbour (other block absent, or outside the grid) replaced by the voxel's
// own normal; FP64 arithmetic on the FP32 normals.
__device__ __forceinline__ void sparse_hessian_voxel(const SpecD& s, int bd, int nbx, int nby,
                                                     const int32_t* __restrict__ ijk,
                                                     const int32_t* __restrict__ table,
                                                     const float4* __restrict__ phin, int blk,
                                                     int local, float* __restrict__ out)
{
    const int V = bd * bd * bd;
    const int lx = local % bd, ly = (local / bd) % bd, lz = local / (bd * bd);
    const int i = ijk[3 * blk] * bd + lx, j = ijk[3 * blk + 1] * bd + ly, k = ijk[3 * blk + 2] * bd + lz;
    if (i >= s.n[0] || j >= s.n[1] || k >= s.n[2])
    {
        for (int q = 0; q < 6; ++q) out[q] = 0.f;
        return;
    }
    const float4 cur = phin[(int64_t)blk * V + local];
    const double curd[3] = {(double)cur.y, (double)cur.z, (double)cur.w};
    auto sample = [&](int ii, int jj, int kk, double n[3]) {
        if (ii < 0 || jj < 0 || kk < 0 || ii >= s.n[0] || jj >= s.n[1] || kk >= s.n[2])
        {
            n[0] = curd[0];
            n[1] = curd[1];
            n[2] = curd[2];
            return;
        }
        const int b2 = table[ii / bd + nbx * (jj / bd + nby * (kk / bd))];
        if (b2 < 0)
        {
            n[0] = curd[0];
            n[1] = curd[1];
            n[2] = curd[2];
            return;
        }
        const int l2 = (ii % bd) + bd * ((jj % bd) + bd * (kk % bd));
        const float4 c = phin[(int64_t)b2 * V + l2];
        n[0] = (double)c.y;
        n[1] = (double)c.z;
        n[2] = (double)c.w;
    };
    double dn[3][3];
    const int off[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int a = 0; a < 3; ++a)
    {
        double pn[3], mn[3];
        sample(i + off[a][0], j + off[a][1], k + off[a][2], pn);
        sample(i - off[a][0], j - off[a][1], k - off[a][2], mn);
        for (int r = 0; r < 3; ++r) dn[a][r] = (pn[r] - mn[r]) / (2.0 * s.voxel[a]);
    }
    double h6[6];
    sym_hessian(dn, h6);
    for (int q = 0; q < 6; ++q) out[q] = (float)h6[q];
}

__global__ void k_sparse_hessian(SpecD s, int bd, int nbx, int nby, int64_t stored,
                                 const int32_t* __restrict__ ijk, const int32_t* __restrict__ table,
                                 const float4* __restrict__ phin, float* __restrict__ hess6)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= stored) return;
    const int V = bd * bd * bd;
    sparse_hessian_voxel(s, bd, nbx, nby, ijk, table, phin, (int)(v / V), (int)(v % V),
                         hess6 + 6 * v);
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
struct Timer
{
    cudaEvent_t e0, e1;
    cudaStream_t s;
    explicit Timer(cudaStream_t st) : s(st)
    {
        SDFO_CUDA(cudaEventCreate(&e0));
        SDFO_CUDA(cudaEventCreate(&e1));
        SDFO_CUDA(cudaEventRecord(e0, s));
    }
    ~Timer()
    {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    double lap()
    {
        SDFO_CUDA(cudaEventRecord(e1, s));
        SDFO_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        SDFO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        SDFO_CUDA(cudaEventRecord(e0, s));
        return ms;
    }
};

// KdTree::rayDirection (KdTree.h:330-333): the fixed vector normalised.
void parity_ray(double dir[3])
{
    const double r[3] = {1.0, 0.3713906763541037, 0.52999894000318};
    volatile double n2 = r[0] * r[0];
    n2 = n2 + r[1] * r[1];
    n2 = n2 + r[2] * r[2];
    const double len = std::sqrt((double)n2);
    for (int a = 0; a < 3; ++a) dir[a] = r[a] / len;
}

// Device-side LBVH with its storage.
struct DeviceLbvh
{
    DeviceBuffer<float4> nodes;
    DeviceBuffer<double> tri9;
    DeviceBuffer<int32_t> tri_id;
    DeviceBuffer<double> pn; // pseudo-normal sign mode only
    int n = 0;
    LbvhView view() const
    {
        LbvhView v{};
        v.nodes = nodes.get();
        v.tri9 = tri9.get();
        v.tri_id = tri_id.get();
        v.n = n;
        parity_ray(v.dir);
        for (int a = 0; a < 3; ++a) v.inv_dir[a] = (float)(1.0 / v.dir[a]);
        v.pn = pn.get();
        v.stackless = lbvh_stackless();
        return v;
    }
};

// Angle-weighted pseudo-normals of a triangle mesh (Baerentzen and Aanaes,
// "Signed distance computation using the angle weighted pseudonormal",
// IEEE TVCG 2005), in FP64, on the device: per triangle the unit face normal
// (none for a degenerate triangle, |cross| <= 1e-15, the face-normal rule);
// per vertex the sum over incident triangles of the corner angle times the
// face normal; per edge the sum of the face normals of the triangles sharing
// it; each normalised.  The corner and edge records are sorted by vertex and
// by edge with a stable radix sort, so every sum runs over its triangles in
// triangle order (deterministic).  For a closed, consistently oriented mesh
// the sign of (p - closest point) . (the normal of the closest point's
// feature) is the inside/outside sign.
__global__ void k_pn_records(const double* __restrict__ verts, const int32_t* __restrict__ tris, int nt,
                             uint32_t* __restrict__ vkey, uint64_t* __restrict__ ekey, int32_t* __restrict__ val,
                             double* __restrict__ fn, double* __restrict__ vcontrib)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const int32_t ix[3] = {tris[3 * (int64_t)t], tris[3 * (int64_t)t + 1], tris[3 * (int64_t)t + 2]};
    d3 P[3];
    for (int k = 0; k < 3; ++k)
        P[k] = mk(verts[3 * (int64_t)ix[k]], verts[3 * (int64_t)ix[k] + 1], verts[3 * (int64_t)ix[k] + 2]);
    const d3 cr = cross(sub(P[1], P[0]), sub(P[2], P[0]));
    const double len = sqrt(dot(cr, cr));
    const bool ok = len > 1e-15;
    const d3 f = ok ? mk(cr.x / len, cr.y / len, cr.z / len) : mk(0.0, 0.0, 0.0);
    fn[3 * (int64_t)t] = f.x;
    fn[3 * (int64_t)t + 1] = f.y;
    fn[3 * (int64_t)t + 2] = f.z;
    const int e[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int k = 0; k < 3; ++k)
    {
        const int64_t r = 3 * (int64_t)t + k;
        vkey[r] = (uint32_t)ix[k];
        val[r] = (int32_t)r;
        const uint32_t a = (uint32_t)ix[e[k][0]], b = (uint32_t)ix[e[k][1]];
        ekey[r] = ((uint64_t)min(a, b) << 32) | max(a, b);
        const d3 u = sub(P[(k + 1) % 3], P[k]), w = sub(P[(k + 2) % 3], P[k]);
        const double lu = sqrt(dot(u, u)), lw = sqrt(dot(w, w));
        double ang = 0.0;
        if (ok && lu > 0.0 && lw > 0.0) ang = acos(fmax(-1.0, fmin(1.0, dot(u, w) / (lu * lw))));
        vcontrib[3 * r] = ang * f.x;
        vcontrib[3 * r + 1] = ang * f.y;
        vcontrib[3 * r + 2] = ang * f.z;
    }
}

__device__ __forceinline__ void put_unit(double* out, double x, double y, double z)
{
    const double l = sqrt(x * x + y * y + z * z);
    out[0] = l > 0.0 ? x / l : 0.0;
    out[1] = l > 0.0 ? y / l : 0.0;
    out[2] = l > 0.0 ? z / l : 0.0;
}

// Vertex normals: the thread at the start of each vertex's run of sorted
// corner records sums the run in order and writes the unit normal for every
// corner of the run (out: 3 doubles per corner record, by record index).
__global__ void k_pn_vertex(int64_t m, const uint32_t* __restrict__ key, const int32_t* __restrict__ val,
                            const double* __restrict__ vcontrib, double* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || (i > 0 && key[i] == key[i - 1])) return;
    double x = 0.0, y = 0.0, z = 0.0;
    int64_t j = i;
    for (; j < m && key[j] == key[i]; ++j)
    {
        const int64_t r = val[j];
        x += vcontrib[3 * r];
        y += vcontrib[3 * r + 1];
        z += vcontrib[3 * r + 2];
    }
    for (int64_t q = i; q < j; ++q) put_unit(out + 3 * (int64_t)val[q], x, y, z);
}

// Edge normals: the same over runs of sorted edge records, summing the face
// normals of the records' triangles.
__global__ void k_pn_edge(int64_t m, const uint64_t* __restrict__ key, const int32_t* __restrict__ val,
                          const double* __restrict__ fn, double* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || (i > 0 && key[i] == key[i - 1])) return;
    double x = 0.0, y = 0.0, z = 0.0;
    int64_t j = i;
    for (; j < m && key[j] == key[i]; ++j)
    {
        const int64_t t = val[j] / 3;
        x += fn[3 * t];
        y += fn[3 * t + 1];
        z += fn[3 * t + 2];
    }
    for (int64_t q = i; q < j; ++q) put_unit(out + 3 * (int64_t)val[q], x, y, z);
}

// Slot-order pseudo-normals: vertex normals of corners a, b, c then edge
// normals of ab, ac, bc of triangle tri_id[slot] (18 doubles per slot).
__global__ void k_pn_assemble(int n, const int32_t* __restrict__ ids, const double* __restrict__ vn,
                              const double* __restrict__ en, double* __restrict__ out)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= 18 * (int64_t)n) return;
    const int64_t s = q / 18, r = q % 18;
    const int64_t t = ids[s];
    out[q] = r < 9 ? vn[9 * t + r] : en[9 * t + (r - 9)];
}

// The pseudo-normals of (verts, tris) (host arrays) in the slot order of a
// tree whose slot -> triangle map is `tri_id` (device).
void upload_pseudo_normals(DeviceBuffer<double>& pn, const double* verts, int64_t nv, const int32_t* tris,
                           int64_t nt, const int32_t* tri_id, cudaStream_t s)
{
    const int64_t m = 3 * nt;
    DeviceBuffer<double> dverts((size_t)nv * 3);
    DeviceBuffer<int32_t> dtris((size_t)m);
    SDFO_CUDA(cudaMemcpyAsync(dverts.get(), verts, sizeof(double) * 3 * (size_t)nv, cudaMemcpyHostToDevice, s));
    SDFO_CUDA(cudaMemcpyAsync(dtris.get(), tris, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice, s));
    DeviceBuffer<uint32_t> vkey((size_t)m), vkey2((size_t)m);
    DeviceBuffer<uint64_t> ekey((size_t)m), ekey2((size_t)m);
    DeviceBuffer<int32_t> val((size_t)m), vval((size_t)m), eval((size_t)m);
    DeviceBuffer<double> fn((size_t)nt * 3), vcontrib((size_t)m * 3), vn((size_t)m * 3), en((size_t)m * 3);
    const int T = 256;
    k_pn_records<<<(unsigned)((nt + T - 1) / T), T, 0, s>>>(dverts.get(), dtris.get(), (int)nt, vkey.get(),
                                                           ekey.get(), val.get(), fn.get(), vcontrib.get());
    SDFO_CHECK_LAUNCH();
    int vbits = 1;
    while (vbits < 32 && (int64_t(1) << vbits) < nv) ++vbits;
    size_t t1 = 0, t2 = 0;
    SDFO_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t1, vkey.get(), vkey2.get(), val.get(), vval.get(), (int)m,
                                              0, vbits, s));
    SDFO_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t2, ekey.get(), ekey2.get(), val.get(), eval.get(), (int)m,
                                              0, 32 + vbits, s));
    DeviceBuffer<unsigned char> tmp(std::max(t1, t2));
    SDFO_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), t1, vkey.get(), vkey2.get(), val.get(), vval.get(), (int)m,
                                              0, vbits, s));
    SDFO_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), t2, ekey.get(), ekey2.get(), val.get(), eval.get(), (int)m,
                                              0, 32 + vbits, s));
    k_pn_vertex<<<(unsigned)((m + T - 1) / T), T, 0, s>>>(m, vkey2.get(), vval.get(), vcontrib.get(), vn.get());
    SDFO_CHECK_LAUNCH();
    k_pn_edge<<<(unsigned)((m + T - 1) / T), T, 0, s>>>(m, ekey2.get(), eval.get(), fn.get(), en.get());
    SDFO_CHECK_LAUNCH();
    pn.reset((size_t)nt * 18);
    k_pn_assemble<<<(unsigned)((18 * nt + T - 1) / T), T, 0, s>>>((int)nt, tri_id, vn.get(), en.get(), pn.get());
    SDFO_CHECK_LAUNCH();
    SDFO_CUDA(cudaStreamSynchronize(s)); // the temporaries are released on return
}

// Host build of the reference's tree (KdTree::build / buildRecursive,
// KdTree.h:91-121, 188-242): median split of the centroids on the longest
// centroid-extent axis with std::nth_element, leaves of <= 8 triangles, nodes
// numbered in creation (pre-)order.  Restated because tie resolution of the
// nearest search (and with it the face-normal sign fallback) depends on this
// exact tree.
//
// The reference partitions an index array whose comparator reads the
// centroid arrays; here the partition runs over 32-byte records {centroid,
// triangle id} kept contiguous, so every pass streams through memory instead
// of gathering.  std::nth_element makes the same comparisons and the same
// moves whatever the element type, so the permutation of triangle ids -- and
// the tree -- is the same as with the index array.  Node boxes are
// unions of the children's boxes, computed after the children: min and max
// are exact, so they equal the reference's min / max over the node's
// triangles.
struct HostRefTree
{
    struct Rec
    {
        double c[3];
        int32_t id;
        int32_t pad;
    };
    RefNode* nodes = nullptr; // subtree_nodes(n) nodes, caller-provided storage
    Rec* rec = nullptr;       // n records, caller-provided storage
    const double* verts = nullptr;
    const int32_t* tris = nullptr;
    std::map<int64_t, int64_t> sizes; // subtree node counts, filled before build

    // Nodes of the subtree over n triangles (leaves of <= 8, median split);
    // the sizes met in one tree take at most two values per level.
    int64_t subtree_nodes(int64_t n)
    {
        if (n <= 8) return 1;
        auto it = sizes.find(n);
        if (it != sizes.end()) return it->second;
        const int64_t v = 1 + subtree_nodes(n / 2) + subtree_nodes(n - n / 2);
        sizes[n] = v;
        return v;
    }

    // Read-only lookup once `sizes` holds every size of the tree.
    int64_t node_count(int64_t n) const
    {
        return n <= 8 ? 1 : sizes.at(n);
    }

    // Node `id` over rec[lo_i, hi_i); children get the pre-order ids id + 1
    // and id + 1 + |left subtree|, so disjoint subtrees can be built
    // concurrently (`depth` levels spawn a thread for the left child).
    void build(int lo_i, int hi_i, int id, int depth)
    {
        RefNode n{};
        n.left = n.right = -1;
        n.start = -1;
        n.count = 0;
        const int count = hi_i - lo_i;
        if (count <= 8)
        {
            // box over the triangles' own boxes (a.cwiseMin(b).cwiseMin(c),
            // a.cwiseMax(b).cwiseMax(c))
            for (int a = 0; a < 3; ++a)
            {
                n.lo[a] = DBL_MAX;
                n.hi[a] = -DBL_MAX;
            }
            for (int i = lo_i; i < hi_i; ++i)
            {
                const int32_t* t = tris + 3 * (size_t)rec[(size_t)i].id;
                const double* A = verts + 3 * (size_t)t[0];
                const double* B = verts + 3 * (size_t)t[1];
                const double* C = verts + 3 * (size_t)t[2];
                for (int a = 0; a < 3; ++a)
                {
                    double mn = B[a] < A[a] ? B[a] : A[a];
                    mn = C[a] < mn ? C[a] : mn;
                    double mx = A[a] < B[a] ? B[a] : A[a];
                    mx = mx < C[a] ? C[a] : mx;
                    n.lo[a] = mn < n.lo[a] ? mn : n.lo[a];
                    n.hi[a] = n.hi[a] < mx ? mx : n.hi[a];
                }
            }
            n.start = lo_i;
            n.count = count;
            nodes[(size_t)id] = n;
            return;
        }
        double cmin[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, cmax[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
        for (int i = lo_i; i < hi_i; ++i)
        {
            const Rec& r = rec[(size_t)i];
            for (int a = 0; a < 3; ++a)
            {
                const double c = r.c[a];
                cmin[a] = c < cmin[a] ? c : cmin[a];
                cmax[a] = cmax[a] < c ? c : cmax[a];
            }
        }
        const double ext[3] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2]};
        int axis = 0;
        if (ext[1] > ext[0]) axis = 1;
        if (ext[2] > ext[axis]) axis = 2;
        const int mid = lo_i + count / 2;
        std::nth_element(rec + lo_i, rec + mid, rec + hi_i,
                         [axis](const Rec& x, const Rec& y) { return x.c[axis] < y.c[axis]; });
        n.left = id + 1;
        n.right = id + 1 + (int)node_count(mid - lo_i);
        if (depth > 0 && count > 4096)
        {
            const int left = n.left;
            std::thread t([this, lo_i, mid, left, depth] { build(lo_i, mid, left, depth - 1); });
            build(mid, hi_i, n.right, depth - 1);
            t.join();
        }
        else
        {
            build(lo_i, mid, n.left, 0);
            build(mid, hi_i, n.right, 0);
        }
        const RefNode& L = nodes[(size_t)n.left];
        const RefNode& R = nodes[(size_t)n.right];
        for (int a = 0; a < 3; ++a)
        {
            n.lo[a] = R.lo[a] < L.lo[a] ? R.lo[a] : L.lo[a];
            n.hi[a] = L.hi[a] < R.hi[a] ? R.hi[a] : L.hi[a];
        }
        nodes[(size_t)id] = n;
    }
};

// Runs body(lo, hi) over [0, n) on up to `threads` host threads.
template <class F>
void host_parallel_for(size_t n, unsigned threads, F&& body)
{
    const size_t min_chunk = 65536;
    threads = (unsigned)std::max<size_t>(1, std::min<size_t>(threads, (n + min_chunk - 1) / min_chunk));
    if (threads <= 1)
    {
        body(size_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    const size_t step = (n + threads - 1) / threads;
    for (unsigned t = 1; t < threads; ++t)
    {
        const size_t lo = std::min(n, t * step), hi = std::min(n, lo + step);
        pool.emplace_back([&body, lo, hi] { body(lo, hi); });
    }
    body(size_t(0), std::min(n, step));
    for (auto& th : pool) th.join();
}

struct DeviceRefTree
{
    DeviceBuffer<RefNode> nodes;
    DeviceBuffer<double> tri9;
    DeviceBuffer<int32_t> tri_id;
    DeviceBuffer<float4> tbox;
    DeviceBuffer<double> pn; // pseudo-normal sign mode only
    int n = 0;
    int nnodes = 0;
    double extent = 1.0;
    RefTreeView view() const
    {
        RefTreeView v{};
        v.nodes = nodes.get();
        v.tri9 = tri9.get();
        v.tri_id = tri_id.get();
        v.n = n;
        v.nnodes = nnodes;
        parity_ray(v.dir);
        v.tbox = triangle_cull() ? tbox.get() : nullptr;
        set_cull_margins(v, extent);
        v.pn = pn.get();
        return v;
    }
};

// The reference tree of one mesh on the host: nodes, triangles in slot order
// (9 doubles each) and slot -> triangle index.
struct HostTreeData
{
    std::vector<RefNode> nodes;
    std::vector<double> tri9;
    std::vector<int32_t> tri_id;
};

// The records of every triangle (centroid (a + b + c) / 3, summed left to
// right as the reference's Eigen expression does; the host code is compiled
// without contraction or reassociation) and the tree over them, into the
// storage h.rec (nt records) and h.nodes (h.subtree_nodes(nt) nodes).
// `threads`: host threads the build may use (0: all of the machine's).
void host_tree_core(HostRefTree& h, const double* verts, const int32_t* tris, int64_t nt, unsigned threads)
{
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    const size_t n = (size_t)nt;
    h.verts = verts;
    h.tris = tris;
    host_parallel_for(n, threads, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i)
        {
            const double* a = verts + 3 * (size_t)tris[3 * i];
            const double* b = verts + 3 * (size_t)tris[3 * i + 1];
            const double* c = verts + 3 * (size_t)tris[3 * i + 2];
            HostRefTree::Rec& r = h.rec[i];
            for (int q = 0; q < 3; ++q) r.c[q] = (a[q] + b[q] + c[q]) / 3.0;
            r.id = (int32_t)i;
            r.pad = 0;
        }
    });
    // up to 2^depth subtrees built concurrently (disjoint ranges of `rec`)
    int depth = 0;
    while (depth < 4 && (2u << depth) <= threads) ++depth;
    h.build(0, (int)nt, 0, depth);
}

// The reference tree of one mesh on the host, with the slot order and (if
// with_tri9) the triangles in slot order.
void host_ref_tree(HostTreeData& out, const double* verts, const int32_t* tris, int64_t nt,
                   unsigned threads = 0, bool with_tri9 = true)
{
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    const size_t n = (size_t)nt;
    HostRefTree h;
    std::vector<HostRefTree::Rec> rec(n);
    out.nodes.resize((size_t)h.subtree_nodes(nt));
    h.rec = rec.data();
    h.nodes = out.nodes.data();
    host_tree_core(h, verts, tris, nt, threads);
    out.tri9.resize(with_tri9 ? 9 * n : 0);
    out.tri_id.resize(n);
    host_parallel_for(n, threads, [&](size_t lo, size_t hi) {
        for (size_t sl = lo; sl < hi; ++sl)
        {
            const int32_t ti = rec[sl].id;
            out.tri_id[sl] = ti;
            if (!with_tri9) continue;
            for (int v = 0; v < 3; ++v)
                for (int q = 0; q < 3; ++q)
                    out.tri9[9 * sl + 3 * v + q] = verts[3 * (size_t)tris[3 * (size_t)ti + v] + q];
        }
    });
}

// Host memory reused by single-mesh tree builds: the records, and a pinned
// block holding the nodes and the slot order so that they upload at copy
// bandwidth and fresh pages are not faulted in on every build.  Builds that
// run at the same time take turns on it.
struct TreeStaging
{
    std::mutex mu;
    std::vector<HostRefTree::Rec> rec;
    unsigned char* pinned = nullptr;
    size_t pinned_bytes = 0;
};

TreeStaging& tree_staging()
{
    static TreeStaging* st = new TreeStaging(); // never destroyed: kept for the process
    return *st;
}

__global__ void k_gather_tri9(const double* __restrict__ verts, const int32_t* __restrict__ tris,
                              const int32_t* __restrict__ ids, int n, double* __restrict__ tri9)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int t = ids[s];
    for (int v = 0; v < 3; ++v)
    {
        const int vi = tris[3 * (int64_t)t + v];
        for (int a = 0; a < 3; ++a) tri9[9 * (int64_t)s + 3 * v + a] = verts[3 * (int64_t)vi + a];
    }
}

void build_ref_tree(DeviceRefTree& t, const double* verts, int64_t nv, const int32_t* tris, int64_t nt,
                    double extent, cudaStream_t s)
{
    t.extent = extent;
    const size_t n = (size_t)nt;
    HostRefTree h;
    const size_t nnodes = (size_t)h.subtree_nodes(nt);
    const size_t node_bytes = sizeof(RefNode) * nnodes;
    const size_t need = node_bytes + sizeof(int32_t) * n;
    TreeStaging& st = tree_staging();
    std::lock_guard<std::mutex> lock(st.mu);
    if (st.pinned_bytes < need)
    {
        if (st.pinned) cudaFreeHost(st.pinned);
        st.pinned = nullptr;
        st.pinned_bytes = 0;
        const size_t want = need + need / 4;
        SDFO_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&st.pinned), want, cudaHostAllocDefault));
        st.pinned_bytes = want;
    }
    if (st.rec.size() < n) st.rec.resize(n);
    h.rec = st.rec.data();
    h.nodes = reinterpret_cast<RefNode*>(st.pinned);
    const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    host_tree_core(h, verts, tris, nt, threads);
    int32_t* ids = reinterpret_cast<int32_t*>(st.pinned + node_bytes);
    host_parallel_for(n, threads, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) ids[i] = st.rec[i].id;
    });
    t.n = (int)nt;
    t.nnodes = (int)nnodes;
    t.nodes.reset(nnodes);
    t.tri9.reset(9 * n);
    t.tri_id.reset(n);
    DeviceBuffer<double> dverts((size_t)nv * 3);
    DeviceBuffer<int32_t> dtris(n * 3);
    SDFO_CUDA(cudaMemcpyAsync(t.nodes.get(), st.pinned, node_bytes, cudaMemcpyHostToDevice, s));
    SDFO_CUDA(cudaMemcpyAsync(t.tri_id.get(), ids, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    SDFO_CUDA(cudaMemcpyAsync(dverts.get(), verts, sizeof(double) * 3 * (size_t)nv, cudaMemcpyHostToDevice, s));
    SDFO_CUDA(cudaMemcpyAsync(dtris.get(), tris, sizeof(int32_t) * 3 * n, cudaMemcpyHostToDevice, s));
    k_gather_tri9<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dverts.get(), dtris.get(), t.tri_id.get(), (int)nt,
                                                             t.tri9.get());
    SDFO_CHECK_LAUNCH();
    t.tbox.reset(2 * n);
    k_tri_boxes<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(t.tri9.get(), (int)nt, t.tbox.get());
    SDFO_CHECK_LAUNCH();
    // the staging block is reused by the next build and the temporaries are
    // freed on return: finish the copies and the gather first
    SDFO_CUDA(cudaStreamSynchronize(s));
}

void build_lbvh(DeviceLbvh& bvh, const double* h_verts, int64_t nv, const int32_t* h_tris, int64_t nt,
               double extent, cudaStream_t s)
{
    const int n = (int)nt;
    bvh.n = n;
    DeviceBuffer<double> verts((size_t)nv * 3);
    DeviceBuffer<int32_t> tris((size_t)nt * 3);
    SDFO_CUDA(cudaMemcpyAsync(verts.get(), h_verts, sizeof(double) * 3 * nv, cudaMemcpyHostToDevice, s));
    SDFO_CUDA(cudaMemcpyAsync(tris.get(), h_tris, sizeof(int32_t) * 3 * nt, cudaMemcpyHostToDevice, s));
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a)
        {
            lo[a] = std::min(lo[a], h_verts[3 * i + a]);
            hi[a] = std::max(hi[a], h_verts[3 * i + a]);
        }
    double ie[3];
    for (int a = 0; a < 3; ++a) ie[a] = hi[a] > lo[a] ? 1.0 / (hi[a] - lo[a]) : 0.0;
    DeviceBuffer<uint64_t> keys(nt), keys_sorted(nt);
    DeviceBuffer<int32_t> ids(nt);
    bvh.tri_id.reset(nt);
    const int T = 256;
    k_morton<<<(n + T - 1) / T, T, 0, s>>>(verts.get(), tris.get(), n, make_double3(lo[0], lo[1], lo[2]),
                                           make_double3(ie[0], ie[1], ie[2]), keys.get(), ids.get());
    SDFO_CHECK_LAUNCH();
    size_t temp = 0;
    SDFO_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys.get(), keys_sorted.get(), ids.get(),
                                              bvh.tri_id.get(), n, 0, 63, s));
    DeviceBuffer<unsigned char> tmp(temp);
    SDFO_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), temp, keys.get(), keys_sorted.get(), ids.get(),
                                              bvh.tri_id.get(), n, 0, 63, s));
    bvh.tri9.reset((size_t)nt * 9);
    DeviceBuffer<double> box64((size_t)(2 * n - 1) * 6);
    k_gather_tris<<<(n + T - 1) / T, T, 0, s>>>(verts.get(), tris.get(), bvh.tri_id.get(), n,
                                                bvh.tri9.get(), box64.get());
    SDFO_CHECK_LAUNCH();
    if (n == 1) return;
    DeviceBuffer<int2> children((size_t)(n - 1));
    DeviceBuffer<int32_t> parent((size_t)(2 * n - 1));
    DeviceBuffer<int> arrivals((size_t)(n - 1));
    SDFO_CUDA(cudaMemsetAsync(arrivals.get(), 0, sizeof(int) * (n - 1), s));
    SDFO_CUDA(cudaMemsetAsync(parent.get(), 0xff, sizeof(int32_t) * (2 * n - 1), s));
    k_karras<<<(n - 1 + T - 1) / T, T, 0, s>>>(keys_sorted.get(), n, children.get(), parent.get());
    SDFO_CHECK_LAUNCH();
    k_refit<<<(n + T - 1) / T, T, 0, s>>>(n, children.get(), parent.get(), arrivals.get(), box64.get());
    SDFO_CHECK_LAUNCH();
    bvh.nodes.reset((size_t)(n - 1) * 4);
    const double margin = 4.0e-6 * extent;
    k_pack<<<(n - 1 + T - 1) / T, T, 0, s>>>(n, children.get(), parent.get(), box64.get(), margin,
                                             bvh.nodes.get());
    SDFO_CHECK_LAUNCH();
}

// The acceleration structure selected by sdfo_set_bvh_mode, with the
// pseudo-normals when sdfo_set_sign_mode selects that sign.
struct AnyTree
{
    int mode;
    DeviceRefTree ref;
    DeviceLbvh lbvh;
    void build(const double* verts, int64_t nv, const int32_t* tris, int64_t nt, double extent,
               cudaStream_t s)
    {
        const bool pseudo = sign_mode() == SDFO_SIGN_PSEUDONORMAL;
        if (mode == SDFO_BVH_LBVH)
        {
            build_lbvh(lbvh, verts, nv, tris, nt, extent, s);
            if (pseudo) upload_pseudo_normals(lbvh.pn, verts, nv, tris, nt, lbvh.tri_id.get(), s);
        }
        else
        {
            build_ref_tree(ref, verts, nv, tris, nt, extent, s);
            if (pseudo) upload_pseudo_normals(ref.pn, verts, nv, tris, nt, ref.tri_id.get(), s);
        }
    }
    int node_count(int64_t nt) const
    {
        return mode == SDFO_BVH_LBVH ? (int)(nt > 1 ? nt - 1 : 0) : ref.nnodes;
    }
    template <class F>
    void visit(F&& f) const
    {
        if (mode == SDFO_BVH_LBVH)
            f(lbvh.view());
        else
            f(ref.view());
    }
};

// Threads per CTA of a one-candidate-per-thread launch over `total`
// candidates: 256, or fewer (a multiple of 32, at least 32) so that small
// launches still spread over two CTAs per SM instead of a handful of SMs
// (the hollow cylinder's 2,048 candidate blocks: 64 CTAs of 32, not 8 of 256).
int spread_threads(int64_t total)
{
    const int64_t want = 2 * (int64_t)current_sm_count();
    int t = 256;
    while (t > 32 && (total + t - 1) / t < want) t -= 32;
    return t;
}

double scene_extent(const double* verts, int64_t nv, const sdfo_grid_info& info)
{
    double e = 0.0;
    for (int64_t i = 0; i < 3 * nv; ++i) e = std::max(e, std::fabs(verts[i]));
    for (int a = 0; a < 3; ++a) e = std::max({e, std::fabs(info.bmin[a]), std::fabs(info.bmax[a])});
    return e > 0.0 ? e : 1.0;
}

SpecD spec_of(const sdfo_grid_info& info)
{
    SpecD s{};
    for (int a = 0; a < 3; ++a)
    {
        s.bmin[a] = info.bmin[a];
        s.voxel[a] = info.voxel[a];
        s.n[a] = info.shape[a];
    }
    return s;
}

void check_status(const DeviceBuffer<int>& status, cudaStream_t s)
{
    int h = 0;
    SDFO_CUDA(cudaMemcpyAsync(&h, status.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    SDFO_CUDA(cudaStreamSynchronize(s));
    if (h & kStatusStackOverflow)
        throw Error(SDFO_ERR_DEVICE_STATUS, "BVH traversal stack overflow (tree deeper than 64)");
}

} // namespace

} // namespace sdfo
