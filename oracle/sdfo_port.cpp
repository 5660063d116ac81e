/*
 * sdfo_port.cpp -- CPU restatement of the SdfOracle hot path (oracle).
 *
 * TEST INFRASTRUCTURE ONLY; see sdfo_port.h.  Compiled with
 * -ffp-contract=off (oracle/Makefile) so every FP64 expression below is
 * evaluated in the order written, which is the reference's order.  Vector
 * sums are left folds ((x0 + x1) + x2), the order Eigen uses for fixed-size
 * 3-vectors.
 */
#include "sdfo_port.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

void port_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* small FP64 vector helpers                                                */
/* ------------------------------------------------------------------------ */

static inline double dot3(const double* a, const double* b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline void sub3(const double* a, const double* b, double* o)
{
    o[0] = a[0] - b[0];
    o[1] = a[1] - b[1];
    o[2] = a[2] - b[2];
}
static inline void cross3(const double* a, const double* b, double* o)
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double norm3(const double* a) { return sqrt(dot3(a, a)); }

/* ------------------------------------------------------------------------ */
/* grid setup: SdfBuilder.cpp:994-1035, GridSpec.h:65-74                    */
/* ------------------------------------------------------------------------ */

int port_snap_resolution(int n, int maxRes)
{
    static const int levels[] = {8, 16, 32, 64, 128, 256, 512, 1024, 2048};
    for (int i = 0; i < 9; ++i)
    {
        const int v = levels[i];
        if (v >= n || v >= maxRes) return v < maxRes ? v : maxRes;
    }
    return maxRes;
}

void port_setup_grid(const double* verts, int nv, double padding, double voxelSize,
                     int targetResolution, int maxResolution, port_grid_spec* out)
{
    double vmin[3] = {1e30, 1e30, 1e30};
    double vmax[3] = {-1e30, -1e30, -1e30};
    for (int i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a)
        {
            const double x = verts[3 * i + a];
            vmin[a] = x < vmin[a] ? x : vmin[a]; /* cwiseMin */
            vmax[a] = vmax[a] < x ? x : vmax[a]; /* cwiseMax */
        }
    double d[3];
    sub3(vmax, vmin, d);
    const double diag = norm3(d);
    const double pad = padding * diag;
    double bmin[3], bmax[3], size[3];
    for (int a = 0; a < 3; ++a)
    {
        bmin[a] = vmin[a] - pad;
        bmax[a] = vmax[a] + pad;
    }
    sub3(bmax, bmin, size);
    double h = voxelSize;
    if (h <= 0.0)
    {
        double longest = size[0];
        if (longest < size[1]) longest = size[1];
        if (longest < size[2]) longest = size[2];
        h = longest / (double)targetResolution;
    }
    for (int a = 0; a < 3; ++a)
    {
        int raw = (int)ceil(size[a] / h);
        if (raw < 1) raw = 1;
        out->shape[a] = port_snap_resolution(raw, maxResolution);
        out->bmin[a] = bmin[a];
        out->voxel[a] = h;
    }
    for (int a = 0; a < 3; ++a) out->bmax[a] = bmin[a] + (double)out->shape[a] * h;
}

static inline void center_from_index(const port_grid_spec* s, int i, int j, int k, double* c)
{
    /* GridSpec::centerFromIndex (GridSpec.h:29-33) */
    c[0] = s->bmin[0] + s->voxel[0] * (i + 0.5);
    c[1] = s->bmin[1] + s->voxel[1] * (j + 0.5);
    c[2] = s->bmin[2] + s->voxel[2] * (k + 0.5);
}

static inline int in_bounds(const port_grid_spec* s, int i, int j, int k)
{
    return i >= 0 && i < s->shape[0] && j >= 0 && j < s->shape[1] && k >= 0 && k < s->shape[2];
}

/* ------------------------------------------------------------------------ */
/* triangle primitives: KdTree.h:26-74, 330-396                             */
/* ------------------------------------------------------------------------ */

/* Ericson's closest point on triangle (Real-Time Collision Detection 5.1.5),
 * with the reference's branch order and arithmetic (KdTree.h:26-74). */
static void closest_point_on_triangle(const double* p, const double* a, const double* b,
                                      const double* c, double* out)
{
    double ab[3], ac[3], ap[3];
    sub3(b, a, ab);
    sub3(c, a, ac);
    sub3(p, a, ap);
    const double d1 = dot3(ab, ap);
    const double d2 = dot3(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0)
    {
        memcpy(out, a, 3 * sizeof(double));
        return;
    }
    double bp[3];
    sub3(p, b, bp);
    const double d3 = dot3(ab, bp);
    const double d4 = dot3(ac, bp);
    if (d3 >= 0.0 && d4 <= d3)
    {
        memcpy(out, b, 3 * sizeof(double));
        return;
    }
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0)
    {
        const double v = d1 / (d1 - d3);
        for (int q = 0; q < 3; ++q) out[q] = a[q] + v * ab[q];
        return;
    }
    double cp[3];
    sub3(p, c, cp);
    const double d5 = dot3(ab, cp);
    const double d6 = dot3(ac, cp);
    if (d6 >= 0.0 && d5 <= d6)
    {
        memcpy(out, c, 3 * sizeof(double));
        return;
    }
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0)
    {
        const double w = d2 / (d2 - d6);
        for (int q = 0; q < 3; ++q) out[q] = a[q] + w * ac[q];
        return;
    }
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0)
    {
        const double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int q = 0; q < 3; ++q) out[q] = b[q] + w * (c[q] - b[q]);
        return;
    }
    const double denom = 1.0 / (va + vb + vc);
    const double v = vb * denom;
    const double w = vc * denom;
    for (int q = 0; q < 3; ++q) out[q] = a[q] + ab[q] * v + ac[q] * w;
}

/* Face normal as the nearest search stores it (KdTree.h:310-314). */
static void face_normal(const double* a, const double* b, const double* c, double* out)
{
    double e1[3], e2[3], n[3];
    sub3(b, a, e1);
    sub3(c, a, e2);
    cross3(e1, e2, n);
    const double len = norm3(n);
    if (len > 1.0e-15)
    {
        for (int q = 0; q < 3; ++q) out[q] = n[q] / len;
    }
    else
    {
        out[0] = 0.0;
        out[1] = 0.0;
        out[2] = 1.0;
    }
}

/* Fixed parity ray (KdTree.h:330-333): (1, 0.3713906763541037,
 * 0.52999894000318).normalized(). */
static void ray_direction(double* d)
{
    const double v[3] = {1.0, 0.3713906763541037, 0.52999894000318};
    const double n2 = dot3(v, v);
    const double n = sqrt(n2);
    for (int q = 0; q < 3; ++q) d[q] = v[q] / n;
}

/* Moller-Trumbore with the reference's tolerances (KdTree.h:362-396). */
static int ray_hits_triangle(const double* o, const double* dir, const double* a,
                             const double* b, const double* c)
{
    const double eps = 1.0e-12;
    double e1[3], e2[3], h[3];
    sub3(b, a, e1);
    sub3(c, a, e2);
    cross3(dir, e2, h);
    const double det = dot3(e1, h);
    if (fabs(det) < eps) return 0;
    const double invDet = 1.0 / det;
    double s[3];
    sub3(o, a, s);
    const double u = invDet * dot3(s, h);
    if (u < -eps || u > 1.0 + eps) return 0;
    double q[3];
    cross3(s, e1, q);
    const double v = invDet * dot3(dir, q);
    if (v < -eps || u + v > 1.0 + eps) return 0;
    const double t = invDet * dot3(e2, q);
    return t > eps;
}

/* ------------------------------------------------------------------------ */
/* the reference's triangle tree (KdTree.h:86-442), restated                */
/* ------------------------------------------------------------------------ */
/* Median split on the longest centroid-extent axis with std::nth_element
 * (KdTree.h:188-242), leaves of <= 8 triangles, nodes in creation (pre-)order.
 * The nearest search visits nodes in the same near-first depth-first order
 * and updates only on a strictly smaller squared distance, so ties resolve to
 * the triangle the reference finds first. */

typedef struct
{
    double lo[3], hi[3];
    int left, right; /* internal */
    int start, count; /* leaf: range in order[] */
} pnode;

struct port_bvh
{
    int nt;
    std::vector<double> tv;  /* (nt, 9) triangle vertices, original order */
    std::vector<double> tlo, thi, cen; /* per-triangle bounds and centroid */
    std::vector<int> order;  /* m_indices */
    std::vector<pnode> nodes;
    double dir[3];
};

static int build_node(port_bvh* b, int lo, int hi)
{
    const int id = (int)b->nodes.size();
    b->nodes.emplace_back();
    double bmin[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, bmax[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    double cmin[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, cmax[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int i = lo; i < hi; ++i)
    {
        const int t = b->order[i];
        for (int a = 0; a < 3; ++a)
        {
            bmin[a] = b->tlo[3 * t + a] < bmin[a] ? b->tlo[3 * t + a] : bmin[a];
            bmax[a] = bmax[a] < b->thi[3 * t + a] ? b->thi[3 * t + a] : bmax[a];
            cmin[a] = b->cen[3 * t + a] < cmin[a] ? b->cen[3 * t + a] : cmin[a];
            cmax[a] = cmax[a] < b->cen[3 * t + a] ? b->cen[3 * t + a] : cmax[a];
        }
    }
    pnode n;
    for (int a = 0; a < 3; ++a)
    {
        n.lo[a] = bmin[a];
        n.hi[a] = bmax[a];
    }
    n.left = n.right = -1;
    n.start = -1;
    n.count = 0;
    const int count = hi - lo;
    if (count <= 8)
    {
        n.start = lo;
        n.count = count;
        b->nodes[id] = n;
        return id;
    }
    const double ext[3] = {cmax[0] - cmin[0], cmax[1] - cmin[1], cmax[2] - cmin[2]};
    int axis = 0;
    if (ext[1] > ext[0]) axis = 1;
    if (ext[2] > ext[axis]) axis = 2;
    const int mid = lo + count / 2;
    const double* cen = b->cen.data();
    std::nth_element(b->order.begin() + lo, b->order.begin() + mid, b->order.begin() + hi,
                     [cen, axis](int x, int y) { return cen[3 * x + axis] < cen[3 * y + axis]; });
    b->nodes[id] = n;
    const int l = build_node(b, lo, mid);
    const int r = build_node(b, mid, hi);
    b->nodes[id].left = l;
    b->nodes[id].right = r;
    return id;
}

port_bvh* port_bvh_build(const double* verts, int nv, const int* tris, int nt)
{
    (void)nv;
    port_bvh* b = new port_bvh();
    b->nt = nt;
    b->tv.resize(9 * (size_t)nt);
    b->tlo.resize(3 * (size_t)nt);
    b->thi.resize(3 * (size_t)nt);
    b->cen.resize(3 * (size_t)nt);
    b->order.resize((size_t)nt);
    for (int t = 0; t < nt; ++t)
    {
        const double* a = verts + 3 * tris[3 * t];
        const double* bb = verts + 3 * tris[3 * t + 1];
        const double* c = verts + 3 * tris[3 * t + 2];
        for (int q = 0; q < 3; ++q)
        {
            b->tv[9 * t + q] = a[q];
            b->tv[9 * t + 3 + q] = bb[q];
            b->tv[9 * t + 6 + q] = c[q];
            /* a.cwiseMin(b).cwiseMin(c), (a + b + c) / 3.0 (KdTree.h:105-111) */
            double mn = bb[q] < a[q] ? bb[q] : a[q];
            mn = c[q] < mn ? c[q] : mn;
            double mx = a[q] < bb[q] ? bb[q] : a[q];
            mx = mx < c[q] ? c[q] : mx;
            b->tlo[3 * t + q] = mn;
            b->thi[3 * t + q] = mx;
            b->cen[3 * t + q] = (a[q] + bb[q] + c[q]) / 3.0;
        }
        b->order[t] = t;
    }
    if (nt > 0)
    {
        b->nodes.reserve(2 * (size_t)nt);
        build_node(b, 0, nt);
    }
    ray_direction(b->dir);
    return b;
}

void port_bvh_free(port_bvh* b) { delete b; }

/* squaredDistanceToAabb (KdTree.h:244-264) */
static inline double box_dist_sq(const double* p, const double* lo, const double* hi)
{
    double sq = 0.0;
    for (int a = 0; a < 3; ++a)
    {
        if (p[a] < lo[a])
        {
            const double d = lo[a] - p[a];
            sq += d * d;
        }
        else if (p[a] > hi[a])
        {
            const double d = p[a] - hi[a];
            sq += d * d;
        }
    }
    return sq;
}

typedef struct
{
    double sq;
    int tri;
    double cp[3];
} nearest_t;

/* Traversal work counted by port_traversal_counts (NULL otherwise): nodes
 * entered past the nearest search's box cut and their closest-point tests;
 * ray-box tests and ray-triangle tests. */
static thread_local int64_t* t_count = NULL;

/* searchNearest (KdTree.h:266-328): near-first depth-first branch and bound. */
static void nearest_rec(const port_bvh* b, int id, const double* p, nearest_t* best)
{
    const pnode* n = &b->nodes[id];
    if (box_dist_sq(p, n->lo, n->hi) > best->sq) return;
    if (t_count) ++t_count[0];
    if (n->count > 0)
    {
        if (t_count) t_count[1] += n->count;
        for (int i = n->start; i < n->start + n->count; ++i)
        {
            const int t = b->order[i];
            const double* tv = b->tv.data() + 9 * t;
            double cp[3], d[3];
            closest_point_on_triangle(p, tv, tv + 3, tv + 6, cp);
            sub3(p, cp, d);
            const double sq = dot3(d, d);
            if (sq < best->sq)
            {
                best->sq = sq;
                best->tri = t;
                memcpy(best->cp, cp, sizeof(cp));
            }
        }
        return;
    }
    const pnode* L = &b->nodes[n->left];
    const pnode* R = &b->nodes[n->right];
    const double dl = box_dist_sq(p, L->lo, L->hi);
    const double dr = box_dist_sq(p, R->lo, R->hi);
    int first = n->left, second = n->right;
    double df = dl, ds = dr;
    if (dr < dl)
    {
        first = n->right;
        second = n->left;
        df = dr;
        ds = dl;
    }
    if (df <= best->sq) nearest_rec(b, first, p, best);
    if (ds <= best->sq) nearest_rec(b, second, p, best);
}

static void nearest(const port_bvh* b, const double* p, nearest_t* best)
{
    best->sq = DBL_MAX;
    best->tri = -1;
    best->cp[0] = best->cp[1] = best->cp[2] = 0.0;
    if (!b->nodes.empty()) nearest_rec(b, 0, p, best);
}

/* rayIntersectsAabb (KdTree.h:335-360) */
static int ray_box(const port_bvh* b, const double* o, const pnode* n)
{
    double tmin = 0.0, tmax = DBL_MAX;
    for (int a = 0; a < 3; ++a)
    {
        const double inv = 1.0 / b->dir[a];
        double t0 = (n->lo[a] - o[a]) * inv;
        double t1 = (n->hi[a] - o[a]) * inv;
        if (t0 > t1)
        {
            const double t = t0;
            t0 = t1;
            t1 = t;
        }
        tmin = tmin < t0 ? t0 : tmin;
        tmax = t1 < tmax ? t1 : tmax;
        if (tmax < tmin) return 0;
    }
    return 1;
}

static int ray_count_rec(const port_bvh* b, int id, const double* o)
{
    const pnode* n = &b->nodes[id];
    if (t_count) ++t_count[2];
    if (!ray_box(b, o, n)) return 0;
    if (n->count > 0)
    {
        if (t_count) t_count[3] += n->count;
        int hits = 0;
        for (int i = n->start; i < n->start + n->count; ++i)
        {
            const double* tv = b->tv.data() + 9 * b->order[i];
            hits += ray_hits_triangle(o, b->dir, tv, tv + 3, tv + 6);
        }
        return hits;
    }
    return ray_count_rec(b, n->left, o) + ray_count_rec(b, n->right, o);
}

static int ray_count(const port_bvh* b, const double* o)
{
    return b->nodes.empty() ? 0 : ray_count_rec(b, 0, o);
}

/* findSignedNearest (KdTree.h:143-165). */
static void signed_nearest_one(const port_bvh* b, const double* p, double* sd, double* cp,
                               double* fn, int* tri, int* hitsOut)
{
    nearest_t best;
    nearest(b, p, &best);
    const double dist = sqrt(best.sq);
    double nrm[3] = {0.0, 0.0, 1.0};
    if (best.tri >= 0)
    {
        const double* tv = b->tv.data() + 9 * best.tri;
        face_normal(tv, tv + 3, tv + 6, nrm);
    }
    const int hits = ray_count(b, p);
    double s;
    if (hits > 0)
    {
        s = (hits % 2) == 1 ? -dist : dist;
    }
    else
    {
        double diff[3];
        sub3(p, best.cp, diff);
        s = dot3(diff, nrm) >= 0.0 ? dist : -dist;
    }
    *sd = s;
    if (cp) memcpy(cp, best.cp, 3 * sizeof(double));
    if (fn) memcpy(fn, nrm, 3 * sizeof(double));
    if (tri) *tri = best.tri;
    if (hitsOut) *hitsOut = hits;
}

void port_signed_nearest(const port_bvh* b, const double* pts, int64_t n, double* sd,
                         double* cp, double* fn, int* tri, int* hits)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i)
        signed_nearest_one(b, pts + 3 * i, sd + i, cp ? cp + 3 * i : NULL, fn ? fn + 3 * i : NULL,
                           tri ? tri + i : NULL, hits ? hits + i : NULL);
}

void port_traversal_counts(const port_bvh* b, const double* pts, int64_t n, int64_t* counts)
{
    counts[0] = counts[1] = counts[2] = counts[3] = 0;
    for (int64_t i = 0; i < n; ++i)
    {
        double sd;
        t_count = counts;
        signed_nearest_one(b, pts + 3 * i, &sd, NULL, NULL, NULL, NULL);
        t_count = NULL;
    }
}

void port_nearest_distance(const port_bvh* b, const double* pts, int64_t n, double* dist)
{
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i)
    {
        nearest_t best;
        nearest(b, pts + 3 * i, &best);
        dist[i] = sqrt(best.sq);
    }
}

/* SdfBuilder.cpp:1063-1085: normal from the closest point, or the face
 * normal within 1e-12 of the surface. */
static void voxel_normal(const double* c, double sd, const double* cp, const double* fn,
                         double* g)
{
    double diff[3];
    sub3(c, cp, diff);
    const double dist = norm3(diff);
    const double sign = sd >= 0.0 ? 1.0 : -1.0;
    if (dist > 1e-12)
    {
        for (int q = 0; q < 3; ++q) g[q] = sign * diff[q] / dist;
    }
    else
    {
        for (int q = 0; q < 3; ++q) g[q] = sign * fn[q];
    }
}

/* ------------------------------------------------------------------------ */
/* dense build: SdfBuilder.cpp:1039-1152                                    */
/* ------------------------------------------------------------------------ */

void port_build_dense(const port_bvh* b, const port_grid_spec* s, double* phi, double* normal,
                      double* hess6, double* witness)
{
    const int nx = s->shape[0], ny = s->shape[1], nz = s->shape[2];
    const int64_t total = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t idx = 0; idx < total; ++idx)
    {
        const int i = (int)(idx % nx);
        const int j = (int)((idx / nx) % ny);
        const int k = (int)(idx / ((int64_t)nx * ny));
        double c[3], sd, cp[3], fn[3], g[3];
        center_from_index(s, i, j, k, c);
        signed_nearest_one(b, c, &sd, cp, fn, NULL, NULL);
        phi[idx] = sd;
        if (witness) memcpy(witness + 3 * idx, cp, sizeof(cp));
        voxel_normal(c, sd, cp, fn, g);
        memcpy(normal + 3 * idx, g, sizeof(g));
    }
    if (hess6) port_dense_hessian(s, normal, hess6);
}

/* Central differences of the normal field, symmetrised (SdfBuilder.cpp:
 * 1105-1152); dn(a) are the 3 columns, H(r,c) = dn(c)[r]. */
static void hessian_from_columns(const double dn[3][3], double* h6)
{
    /* H = 0.5 * (H + H^T); stored xx, xy, xz, yy, yz, zz */
    h6[0] = 0.5 * (dn[0][0] + dn[0][0]);
    h6[1] = 0.5 * (dn[1][0] + dn[0][1]);
    h6[2] = 0.5 * (dn[2][0] + dn[0][2]);
    h6[3] = 0.5 * (dn[1][1] + dn[1][1]);
    h6[4] = 0.5 * (dn[2][1] + dn[1][2]);
    h6[5] = 0.5 * (dn[2][2] + dn[2][2]);
}

void port_dense_hessian(const port_grid_spec* s, const double* normal, double* hess6)
{
    const int nx = s->shape[0], ny = s->shape[1], nz = s->shape[2];
    const int64_t total = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < total; ++idx)
    {
        const int i = (int)(idx % nx);
        const int j = (int)((idx / nx) % ny);
        const int k = (int)(idx / ((int64_t)nx * ny));
        const int ip = i + 1 < nx ? i + 1 : nx - 1, im = i - 1 >= 0 ? i - 1 : 0;
        const int jp = j + 1 < ny ? j + 1 : ny - 1, jm = j - 1 >= 0 ? j - 1 : 0;
        const int kp = k + 1 < nz ? k + 1 : nz - 1, km = k - 1 >= 0 ? k - 1 : 0;
        const double* np[3] = {normal + 3 * (ip + (int64_t)nx * (j + (int64_t)ny * k)),
                               normal + 3 * (i + (int64_t)nx * (jp + (int64_t)ny * k)),
                               normal + 3 * (i + (int64_t)nx * (j + (int64_t)ny * kp))};
        const double* nm[3] = {normal + 3 * (im + (int64_t)nx * (j + (int64_t)ny * k)),
                               normal + 3 * (i + (int64_t)nx * (jm + (int64_t)ny * k)),
                               normal + 3 * (i + (int64_t)nx * (j + (int64_t)ny * km))};
        double dn[3][3];
        for (int a = 0; a < 3; ++a)
            for (int r = 0; r < 3; ++r) dn[a][r] = (np[a][r] - nm[a][r]) / (2.0 * s->voxel[a]);
        hessian_from_columns(dn, hess6 + 6 * idx);
    }
}

/* ------------------------------------------------------------------------ */
/* sparse narrow band: SdfBuilder.cpp:823-983, 1154-1225                    */
/* ------------------------------------------------------------------------ */

int port_sparse_activate(const port_bvh* b, const port_grid_spec* s, int blockDim,
                         int haloVoxels, double bandDistance, uint8_t* active)
{
    /* bandDistance is the resolved half width (params.bandDistance, or
     * bandVoxels * h when that is 0, SdfBuilder.cpp:835-838). */
    double h = s->voxel[0];
    if (h < s->voxel[1]) h = s->voxel[1];
    if (h < s->voxel[2]) h = s->voxel[2];
    const double blockRadius = 0.5 * sqrt(3.0) * (double)blockDim * h;
    const double activation = bandDistance + (double)haloVoxels * h + blockRadius;
    const int nbx = (s->shape[0] + blockDim - 1) / blockDim;
    const int nby = (s->shape[1] + blockDim - 1) / blockDim;
    const int nbz = (s->shape[2] + blockDim - 1) / blockDim;
    const int total = nbx * nby * nbz;
    int count = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : count)
    for (int bl = 0; bl < total; ++bl)
    {
        const int bi = bl % nbx, bj = (bl / nbx) % nby, bk = bl / (nbx * nby);
        const int i0 = bi * blockDim, j0 = bj * blockDim, k0 = bk * blockDim;
        const int i1 = i0 + blockDim < s->shape[0] ? i0 + blockDim : s->shape[0];
        const int j1 = j0 + blockDim < s->shape[1] ? j0 + blockDim : s->shape[1];
        const int k1 = k0 + blockDim < s->shape[2] ? k0 + blockDim : s->shape[2];
        double c[3];
        c[0] = s->bmin[0] + s->voxel[0] * (0.5 * (double)(i0 + i1));
        c[1] = s->bmin[1] + s->voxel[1] * (0.5 * (double)(j0 + j1));
        c[2] = s->bmin[2] + s->voxel[2] * (0.5 * (double)(k0 + k1));
        nearest_t best;
        nearest(b, c, &best);
        const double dist = sqrt(best.sq);
        active[bl] = fabs(dist) <= activation ? 1 : 0;
        count += active[bl];
    }
    return count;
}

void port_sparse_fill(const port_bvh* b, const port_grid_spec* s, int blockDim, int nblocks,
                      const int* ijk, float* phi, float* normal)
{
    const int V = blockDim * blockDim * blockDim;
#pragma omp parallel for schedule(dynamic, 1)
    for (int blk = 0; blk < nblocks; ++blk)
    {
        for (int local = 0; local < V; ++local)
        {
            const int lx = local % blockDim, ly = (local / blockDim) % blockDim,
                      lz = local / (blockDim * blockDim);
            const int i = ijk[3 * blk] * blockDim + lx;
            const int j = ijk[3 * blk + 1] * blockDim + ly;
            const int k = ijk[3 * blk + 2] * blockDim + lz;
            float* ph = phi + (int64_t)blk * V + local;
            float* nn = normal + 3 * ((int64_t)blk * V + local);
            if (!in_bounds(s, i, j, k))
            {
                *ph = 0.0f;
                nn[0] = 1.0f;
                nn[1] = 0.0f;
                nn[2] = 0.0f;
                continue;
            }
            double c[3], sd, cp[3], fn[3], g[3];
            center_from_index(s, i, j, k, c);
            signed_nearest_one(b, c, &sd, cp, fn, NULL, NULL);
            voxel_normal(c, sd, cp, fn, g);
            *ph = (float)sd;
            nn[0] = (float)g[0];
            nn[1] = (float)g[1];
            nn[2] = (float)g[2];
        }
    }
}

typedef struct
{
    const port_grid_spec* s;
    int bd, nbx, nby, nbz;
    int* table; /* dense block-coordinate table -> block index or -1 */
} sparse_index;

static void sparse_index_init(sparse_index* x, const port_grid_spec* s, int bd, int nblocks,
                              const int* ijk)
{
    x->s = s;
    x->bd = bd;
    x->nbx = (s->shape[0] + bd - 1) / bd;
    x->nby = (s->shape[1] + bd - 1) / bd;
    x->nbz = (s->shape[2] + bd - 1) / bd;
    const int64_t tot = (int64_t)x->nbx * x->nby * x->nbz;
    x->table = (int*)malloc(sizeof(int) * (size_t)tot);
    for (int64_t i = 0; i < tot; ++i) x->table[i] = -1;
    for (int b = 0; b < nblocks; ++b)
    {
        const int bi = ijk[3 * b], bj = ijk[3 * b + 1], bk = ijk[3 * b + 2];
        if (bi < 0 || bj < 0 || bk < 0 || bi >= x->nbx || bj >= x->nby || bk >= x->nbz) continue;
        int* slot = &x->table[bi + (int64_t)x->nbx * (bj + (int64_t)x->nby * bk)];
        if (*slot < 0) *slot = b; /* first block wins, as unordered_map::emplace */
    }
}

/* SparseSdfData::blockForVoxel + sampleFromBlock (SdfData.h:224-302):
 * returns the stored-voxel index (block*V + local) or -1. */
static inline int64_t sparse_voxel(const sparse_index* x, int i, int j, int k)
{
    if (!in_bounds(x->s, i, j, k)) return -1;
    const int bd = x->bd;
    const int b = x->table[i / bd + (int64_t)x->nbx * (j / bd + (int64_t)x->nby * (k / bd))];
    if (b < 0) return -1;
    const int local = (i % bd) + bd * ((j % bd) + bd * (k % bd));
    return (int64_t)b * bd * bd * bd + local;
}

void port_sparse_hessian(const port_grid_spec* s, int blockDim, int nblocks, const int* ijk,
                         const float* normal, float* hess6)
{
    sparse_index x;
    sparse_index_init(&x, s, blockDim, nblocks, ijk);
    const int V = blockDim * blockDim * blockDim;
#pragma omp parallel for schedule(dynamic, 1)
    for (int blk = 0; blk < nblocks; ++blk)
    {
        for (int local = 0; local < V; ++local)
        {
            const int lx = local % blockDim, ly = (local / blockDim) % blockDim,
                      lz = local / (blockDim * blockDim);
            const int i = ijk[3 * blk] * blockDim + lx;
            const int j = ijk[3 * blk + 1] * blockDim + ly;
            const int k = ijk[3 * blk + 2] * blockDim + lz;
            float* out = hess6 + 6 * ((int64_t)blk * V + local);
            if (!in_bounds(s, i, j, k)) continue; /* stays as initialised */
            const float* cur = normal + 3 * ((int64_t)blk * V + local);
            const double curd[3] = {(double)cur[0], (double)cur[1], (double)cur[2]};
            const int off[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
            double dn[3][3];
            for (int a = 0; a < 3; ++a)
            {
                double pn[3], mn[3];
                const int64_t vp = sparse_voxel(&x, i + off[a][0], j + off[a][1], k + off[a][2]);
                const int64_t vm = sparse_voxel(&x, i - off[a][0], j - off[a][1], k - off[a][2]);
                for (int r = 0; r < 3; ++r)
                {
                    pn[r] = vp >= 0 ? (double)normal[3 * vp + r] : curd[r];
                    mn[r] = vm >= 0 ? (double)normal[3 * vm + r] : curd[r];
                }
                for (int r = 0; r < 3; ++r) dn[a][r] = (pn[r] - mn[r]) / (2.0 * s->voxel[a]);
            }
            double h6[6];
            hessian_from_columns(dn, h6);
            for (int q = 0; q < 6; ++q) out[q] = (float)h6[q];
        }
    }
    free(x.table);
}

/* ------------------------------------------------------------------------ */
/* queries: SdfOracle.cpp:448-851, 932-1092                                 */
/* ------------------------------------------------------------------------ */

/* Trilinear over 8 corner values (corner c = di + 2 dj + 4 dk), in the
 * reference's arithmetic (SdfOracle.cpp:552-583); also the interpolant's
 * mixed second derivatives (new: used by the backward kernels). */
static void trilinear_eval(const double* cc, double u, double v, double w, const double* h,
                           double* gap, double* grad, double* hess)
{
    const double c000 = cc[0], c100 = cc[1], c010 = cc[2], c110 = cc[3];
    const double c001 = cc[4], c101 = cc[5], c011 = cc[6], c111 = cc[7];
    const double c00 = c000 * (1 - u) + c100 * u;
    const double c10 = c010 * (1 - u) + c110 * u;
    const double c01 = c001 * (1 - u) + c101 * u;
    const double c11 = c011 * (1 - u) + c111 * u;
    const double c0 = c00 * (1 - v) + c10 * v;
    const double c1 = c01 * (1 - v) + c11 * v;
    *gap = c0 * (1 - w) + c1 * w;
    grad[0] = ((c100 - c000) * (1 - v) * (1 - w) + (c110 - c010) * v * (1 - w) +
               (c101 - c001) * (1 - v) * w + (c111 - c011) * v * w) / h[0];
    grad[1] = ((c010 - c000) * (1 - u) * (1 - w) + (c110 - c100) * u * (1 - w) +
               (c011 - c001) * (1 - u) * w + (c111 - c101) * u * w) / h[1];
    grad[2] = ((c001 - c000) * (1 - u) * (1 - v) + (c101 - c100) * u * (1 - v) +
               (c011 - c010) * (1 - u) * v + (c111 - c110) * u * v) / h[2];
    if (hess)
    {
        /* d2/du dv = sum over w-weights of the x-y cross differences, etc. */
        const double duv = ((c110 - c010) - (c100 - c000)) * (1 - w) +
                           ((c111 - c011) - (c101 - c001)) * w;
        const double duw = ((c101 - c001) - (c100 - c000)) * (1 - v) +
                           ((c111 - c011) - (c110 - c010)) * v;
        const double dvw = ((c011 - c001) - (c010 - c000)) * (1 - u) +
                           ((c111 - c101) - (c110 - c100)) * u;
        hess[0] = 0.0;
        hess[4] = 0.0;
        hess[8] = 0.0;
        hess[1] = hess[3] = duv / (h[0] * h[1]);
        hess[2] = hess[6] = duw / (h[0] * h[2]);
        hess[5] = hess[7] = dvw / (h[1] * h[2]);
    }
}

static inline double H00(double t) { return t * t * (2.0 * t - 3.0) + 1.0; }
static inline double H10(double t) { return t * (t * (t - 2.0) + 1.0); }
static inline double H01(double t) { return t * t * (3.0 - 2.0 * t); }
static inline double H11(double t) { return t * t * (t - 1.0); }
static inline double D00(double t) { return 6.0 * t * (t - 1.0); }
static inline double D10(double t) { return t * (3.0 * t - 4.0) + 1.0; }
static inline double D01(double t) { return 6.0 * t * (1.0 - t); }
static inline double D11(double t) { return t * (3.0 * t - 2.0); }
/* second derivatives of the cubic Hermite basis (new; for the Hessian) */
static inline double S00(double t) { return 12.0 * t - 6.0; }
static inline double S10(double t) { return 6.0 * t - 4.0; }
static inline double S01(double t) { return 6.0 - 12.0 * t; }
static inline double S11(double t) { return 6.0 * t - 2.0; }

/* Tensor Hermite over the 8 corners with values phi and slopes n*h
 * (SdfOracle.cpp:958-1082), in the reference's summation order. */
static void tricubic_eval(const double* phi, const double* nrm, double u, double v, double w,
                          const double* h, double* gap, double* grad, double* hess)
{
    double gx[8], gy[8], gz[8];
    for (int c = 0; c < 8; ++c)
    {
        gx[c] = nrm[3 * c + 0] * h[0];
        gy[c] = nrm[3 * c + 1] * h[1];
        gz[c] = nrm[3 * c + 2] * h[2];
    }
    const double a[4] = {H00(u), H10(u), H01(u), H11(u)};
    const double b[4] = {H00(v), H10(v), H01(v), H11(v)};
    const double cc[4] = {H00(w), H10(w), H01(w), H11(w)};
    const double da[4] = {D00(u), D10(u), D01(u), D11(u)};
    const double db[4] = {D00(v), D10(v), D01(v), D11(v)};
    const double dc[4] = {D00(w), D10(w), D01(w), D11(w)};
    double g = 0.0, fu = 0.0, fv = 0.0, fw = 0.0;
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di)
            {
                const int c = di + 2 * dj + 4 * dk;
                const double p0 = a[2 * di], p1 = a[2 * di + 1];
                const double q0 = b[2 * dj], q1 = b[2 * dj + 1];
                const double r0 = cc[2 * dk], r1 = cc[2 * dk + 1];
                g += (p0 * q0 * r0) * phi[c];
                g += (p1 * q0 * r0) * gx[c];
                g += (p0 * q1 * r0) * gy[c];
                g += (p0 * q0 * r1) * gz[c];
            }
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di)
            {
                const int c = di + 2 * dj + 4 * dk;
                const double p0 = a[2 * di], p1 = a[2 * di + 1];
                const double dp0 = da[2 * di], dp1 = da[2 * di + 1];
                const double q0 = b[2 * dj], q1 = b[2 * dj + 1];
                const double r0 = cc[2 * dk], r1 = cc[2 * dk + 1];
                (void)p0;
                (void)p1;
                fu += (dp0 * q0 * r0) * phi[c];
                fu += (dp1 * q0 * r0) * gx[c];
                fu += (dp0 * q1 * r0) * gy[c];
                fu += (dp0 * q0 * r1) * gz[c];
            }
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di)
            {
                const int c = di + 2 * dj + 4 * dk;
                const double p0 = a[2 * di], p1 = a[2 * di + 1];
                const double q0 = b[2 * dj], q1 = b[2 * dj + 1];
                const double dq0 = db[2 * dj], dq1 = db[2 * dj + 1];
                const double r0 = cc[2 * dk], r1 = cc[2 * dk + 1];
                (void)q0;
                fv += (p0 * dq0 * r0) * phi[c];
                fv += (p1 * dq0 * r0) * gx[c];
                fv += (p0 * dq1 * r0) * gy[c];
                fv += (p0 * dq0 * r1) * gz[c];
            }
    for (int dk = 0; dk < 2; ++dk)
        for (int dj = 0; dj < 2; ++dj)
            for (int di = 0; di < 2; ++di)
            {
                const int c = di + 2 * dj + 4 * dk;
                const double p0 = a[2 * di], p1 = a[2 * di + 1];
                const double q0 = b[2 * dj], q1 = b[2 * dj + 1];
                const double r0 = cc[2 * dk], r1 = cc[2 * dk + 1];
                const double dr0 = dc[2 * dk], dr1 = dc[2 * dk + 1];
                (void)r0;
                fw += (p0 * q0 * dr0) * phi[c];
                fw += (p1 * q0 * dr0) * gx[c];
                fw += (p0 * q1 * dr0) * gy[c];
                fw += (p0 * q0 * dr1) * gz[c];
            }
    *gap = g;
    grad[0] = fu / h[0];
    grad[1] = fv / h[1];
    grad[2] = fw / h[2];
    if (hess)
    {
        const double sa[4] = {S00(u), S10(u), S01(u), S11(u)};
        const double sb[4] = {S00(v), S10(v), S01(v), S11(v)};
        const double sc[4] = {S00(w), S10(w), S01(w), S11(w)};
        /* X[axis-basis-set]: basis per axis for each of the 6 second
         * derivatives: uu, uv, uw, vv, vw, ww */
        const double* setA[6] = {sa, da, da, a, a, a};
        const double* setB[6] = {b, db, b, sb, db, b};
        const double* setC[6] = {cc, cc, dc, cc, dc, sc};
        double d2[6];
        for (int m = 0; m < 6; ++m)
        {
            double s = 0.0;
            for (int c = 0; c < 8; ++c)
            {
                const int di = c & 1, dj = (c >> 1) & 1, dk = c >> 2;
                const double p0 = setA[m][2 * di], p1 = setA[m][2 * di + 1];
                const double q0 = setB[m][2 * dj], q1 = setB[m][2 * dj + 1];
                const double r0 = setC[m][2 * dk], r1 = setC[m][2 * dk + 1];
                s += (p0 * q0 * r0) * phi[c] + (p1 * q0 * r0) * gx[c] + (p0 * q1 * r0) * gy[c] +
                     (p0 * q0 * r1) * gz[c];
            }
            d2[m] = s;
        }
        hess[0] = d2[0] / (h[0] * h[0]);
        hess[1] = hess[3] = d2[1] / (h[0] * h[1]);
        hess[2] = hess[6] = d2[2] / (h[0] * h[2]);
        hess[4] = d2[3] / (h[1] * h[1]);
        hess[5] = hess[7] = d2[4] / (h[1] * h[2]);
        hess[8] = d2[5] / (h[2] * h[2]);
    }
}

static void unit_or_x(const double* g, double* u)
{
    const double len = norm3(g);
    if (len > 1e-15)
    {
        for (int q = 0; q < 3; ++q) u[q] = g[q] / len;
    }
    else
    {
        u[0] = 1.0;
        u[1] = 0.0;
        u[2] = 0.0;
    }
}

/* Corner fetch callback: returns 0 when a corner is missing. */
typedef int (*corner_fn)(const void* ctx, int i, int j, int k, double* phi, double* n,
                         double* h6);

static void query_one(const port_grid_spec* s, int mode, int hasHessian, corner_fn fetch,
                      const void* ctx, const double* p, double* gapO, double* gradO,
                      double* unitO, double* witO, uint8_t* validO, double* hessO)
{
    double gap = 0.0, grad[3] = {0.0, 0.0, 0.0}, unit[3] = {1.0, 0.0, 0.0}, hs[9] = {0};
    int valid = 0;
    if (mode == PORT_FIRST_ORDER || mode == PORT_SECOND_ORDER)
    {
        /* indexFromWorld (GridSpec.h:37-45) */
        double f[3];
        for (int a = 0; a < 3; ++a) f[a] = (p[a] - s->bmin[a]) / s->voxel[a] - 0.5;
        const int i = (int)round(f[0]), j = (int)round(f[1]), k = (int)round(f[2]);
        double ph, n[3], h6[6];
        const int second = mode == PORT_SECOND_ORDER && hasHessian;
        if (fetch(ctx, i, j, k, &ph, n, second ? h6 : NULL))
        {
            double c[3], dx[3];
            center_from_index(s, i, j, k, c);
            sub3(p, c, dx);
            valid = 1;
            if (!second)
            {
                /* firstOrderQuery (SdfOracle.cpp:494-520) */
                gap = ph + dot3(n, dx);
                memcpy(grad, n, sizeof(grad));
                memcpy(unit, n, sizeof(unit));
            }
            else
            {
                /* secondOrderQuery (SdfOracle.cpp:448-490) */
                const double H[9] = {h6[0], h6[1], h6[2], h6[1], h6[3], h6[4], h6[2], h6[4], h6[5]};
                double row[3];
                for (int cc = 0; cc < 3; ++cc)
                    row[cc] = (0.5 * dx[0]) * H[0 * 3 + cc] + (0.5 * dx[1]) * H[1 * 3 + cc] +
                              (0.5 * dx[2]) * H[2 * 3 + cc];
                const double second_term = row[0] * dx[0] + row[1] * dx[1] + row[2] * dx[2];
                const double first_term = dot3(n, dx);
                gap = ph + first_term + second_term;
                double upd[3];
                for (int r = 0; r < 3; ++r)
                    upd[r] = n[r] + (H[3 * r + 0] * dx[0] + H[3 * r + 1] * dx[1] + H[3 * r + 2] * dx[2]);
                const double len = norm3(upd);
                memcpy(grad, upd, sizeof(grad));
                if (len > 1e-15)
                    for (int q = 0; q < 3; ++q) unit[q] = upd[q] / len;
                else
                    memcpy(unit, n, sizeof(unit));
                memcpy(hs, H, sizeof(hs));
            }
        }
    }
    else
    {
        double f[3];
        for (int a = 0; a < 3; ++a) f[a] = (p[a] - s->bmin[a]) / s->voxel[a] - 0.5;
        const int i0 = (int)floor(f[0]), j0 = (int)floor(f[1]), k0 = (int)floor(f[2]);
        const double u = f[0] - i0, v = f[1] - j0, w = f[2] - k0;
        if (!(i0 < 0 || i0 + 1 >= s->shape[0] || j0 < 0 || j0 + 1 >= s->shape[1] || k0 < 0 ||
              k0 + 1 >= s->shape[2]))
        {
            double ph[8], nn[24];
            int ok = 1;
            for (int c = 0; c < 8 && ok; ++c)
                ok = fetch(ctx, i0 + (c & 1), j0 + ((c >> 1) & 1), k0 + (c >> 2), &ph[c], &nn[3 * c],
                           NULL);
            if (ok)
            {
                valid = 1;
                if (mode == PORT_TRILINEAR)
                    trilinear_eval(ph, u, v, w, s->voxel, &gap, grad, hs);
                else
                    tricubic_eval(ph, nn, u, v, w, s->voxel, &gap, grad, hs);
                unit_or_x(grad, unit);
            }
        }
    }
    if (!valid)
    {
        /* SdfQueryResult defaults: gap 0, normal UnitX, witness 0 */
        gap = 0.0;
        grad[0] = grad[1] = grad[2] = 0.0;
        unit[0] = 1.0;
        unit[1] = unit[2] = 0.0;
        memset(hs, 0, sizeof(hs));
    }
    if (gapO) *gapO = gap;
    if (gradO) memcpy(gradO, grad, sizeof(grad));
    if (unitO) memcpy(unitO, unit, sizeof(unit));
    if (witO)
    {
        if (valid)
            for (int q = 0; q < 3; ++q) witO[q] = p[q] - gap * unit[q];
        else
            witO[0] = witO[1] = witO[2] = 0.0;
    }
    if (validO) *validO = (uint8_t)valid;
    if (hessO) memcpy(hessO, hs, sizeof(hs));
}

typedef struct
{
    const port_grid_spec* s;
    const double* phi;
    const double* normal;
    const double* hess6;
} dense_ctx;

static int dense_fetch(const void* cp, int i, int j, int k, double* phi, double* n, double* h6)
{
    const dense_ctx* c = (const dense_ctx*)cp;
    if (!in_bounds(c->s, i, j, k)) return 0;
    const int64_t idx = i + (int64_t)c->s->shape[0] * (j + (int64_t)c->s->shape[1] * k);
    *phi = c->phi[idx];
    for (int q = 0; q < 3; ++q) n[q] = c->normal[3 * idx + q];
    if (h6)
        for (int q = 0; q < 6; ++q) h6[q] = c->hess6 ? c->hess6[6 * idx + q] : 0.0;
    return 1;
}

void port_query_dense(const port_grid_spec* s, const double* phi, const double* normal,
                      const double* hess6, int mode, const double* pts, int64_t n, double* gap,
                      double* grad, double* unit, double* witness, uint8_t* valid, double* hess)
{
    dense_ctx ctx = {s, phi, normal, hess6};
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; ++q)
        query_one(s, mode, 1, dense_fetch, &ctx, pts + 3 * q, gap ? gap + q : NULL,
                  grad ? grad + 3 * q : NULL, unit ? unit + 3 * q : NULL,
                  witness ? witness + 3 * q : NULL, valid ? valid + q : NULL,
                  hess ? hess + 9 * q : NULL);
}

typedef struct
{
    sparse_index x;
    const float* phi;
    const float* normal;
    const float* hess6;
} sparse_ctx;

static int sparse_fetch(const void* cp, int i, int j, int k, double* phi, double* n, double* h6)
{
    const sparse_ctx* c = (const sparse_ctx*)cp;
    const int64_t v = sparse_voxel(&c->x, i, j, k);
    if (v < 0) return 0;
    *phi = (double)c->phi[v];
    for (int q = 0; q < 3; ++q) n[q] = (double)c->normal[3 * v + q];
    if (h6)
    {
        if (!c->hess6) return 0;
        for (int q = 0; q < 6; ++q) h6[q] = (double)c->hess6[6 * v + q];
    }
    return 1;
}

void port_query_sparse(const port_grid_spec* s, int blockDim, int nblocks, const int* ijk,
                       const float* phi, const float* normal, const float* hess6, int mode,
                       const double* pts, int64_t n, double* gap, double* grad, double* unit,
                       double* witness, uint8_t* valid, double* hess)
{
    sparse_ctx ctx;
    sparse_index_init(&ctx.x, s, blockDim, nblocks, ijk);
    ctx.phi = phi;
    ctx.normal = normal;
    ctx.hess6 = hess6;
    const int hasHessian = hess6 != NULL;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; ++q)
        query_one(s, mode, hasHessian, sparse_fetch, &ctx, pts + 3 * q, gap ? gap + q : NULL,
                  grad ? grad + 3 * q : NULL, unit ? unit + 3 * q : NULL,
                  witness ? witness + 3 * q : NULL, valid ? valid + q : NULL,
                  hess ? hess + 9 * q : NULL);
    free(ctx.x.table);
}

/* ======================================================================== */
/* contact-aware build and query (SdfBuilder.cpp:27-359, 416-821;            */
/* SdfOracle.cpp:269-431)                                                    */
/* ======================================================================== */

namespace {

struct ca_tri
{
    double a[3], b[3], c[3];
    double cn[3][3]; /* corner normals */
    double fn[3];    /* face normal */
    double lo[3], hi[3];
};

struct ca_cand
{
    double phi, dist;
    double n[3], w[3];
    int branch;
};

/* normalizedOrDefault (SdfBuilder.cpp:27-43) */
void normalized_or(const double* v, const double* fallback, double* out)
{
    const double nrm = norm3(v);
    if (nrm <= 1.0e-15)
    {
        const double fnrm = norm3(fallback);
        if (fnrm > 1.0e-15)
        {
            for (int a = 0; a < 3; ++a) out[a] = fallback[a] / fnrm;
            return;
        }
        out[0] = 1.0;
        out[1] = 0.0;
        out[2] = 0.0;
        return;
    }
    for (int a = 0; a < 3; ++a) out[a] = v[a] / nrm;
}

const double kUnitX[3] = {1.0, 0.0, 0.0};

/* barycentricOnTriangle (SdfBuilder.cpp:45-67) */
void barycentric(const double* p, const double* a, const double* b, const double* c, double* out)
{
    double v0[3], v1[3], v2[3];
    sub3(b, a, v0);
    sub3(c, a, v1);
    sub3(p, a, v2);
    const double d00 = dot3(v0, v0), d01 = dot3(v0, v1), d11 = dot3(v1, v1);
    const double d20 = dot3(v2, v0), d21 = dot3(v2, v1);
    const double denom = d00 * d11 - d01 * d01;
    if (fabs(denom) <= 1.0e-15)
    {
        out[0] = out[1] = out[2] = 1.0 / 3.0;
        return;
    }
    const double v = (d11 * d20 - d01 * d21) / denom;
    const double w = (d00 * d21 - d01 * d20) / denom;
    out[0] = 1.0 - v - w;
    out[1] = v;
    out[2] = w;
}

/* branchIdFromNormal (SdfBuilder.cpp:114-134): FNV-1a of the normal
 * quantised to 1/4095. */
int branch_id(const double* raw)
{
    double n[3];
    normalized_or(raw, kUnitX, n);
    uint32_t hash = 2166136261u;
    for (int a = 0; a < 3; ++a)
    {
        double v = n[a];
        v = std::max(-1.0, std::min(1.0, v));
        const int32_t q = (int32_t)lround(v * 4095.0);
        hash ^= (uint32_t)q;
        hash *= 16777619u;
    }
    return (int)(1u + (hash & 0x3fffffffu));
}

/* makeContactCandidate (SdfBuilder.cpp:245-266) */
void make_candidate(const double* p, const ca_tri& t, ca_cand& out)
{
    double cp[3], bary[3], raw[3], d[3];
    closest_point_on_triangle(p, t.a, t.b, t.c, cp);
    barycentric(cp, t.a, t.b, t.c, bary);
    for (int a = 0; a < 3; ++a)
        raw[a] = bary[0] * t.cn[0][a] + bary[1] * t.cn[1][a] + bary[2] * t.cn[2][a];
    normalized_or(raw, t.fn, out.n);
    sub3(p, cp, d);
    out.phi = dot3(d, out.n);
    out.dist = norm3(d);
    memcpy(out.w, cp, sizeof(cp));
    out.branch = branch_id(out.n);
}

/* mergeContactCandidate (SdfBuilder.cpp:136-153) */
void merge_candidate(std::vector<ca_cand>& list, const ca_cand& in, double cosMerge)
{
    for (ca_cand& e : list)
    {
        if (dot3(e.n, in.n) >= cosMerge)
        {
            if (fabs(in.phi) < fabs(e.phi)) e = in;
            return;
        }
    }
    list.push_back(in);
}

} // namespace

struct port_ca
{
    port_grid_spec spec;
    std::vector<ca_tri> tris;
    port_bvh* tree = nullptr;
    int tileDim = 8, tnx = 1, tny = 1, tnz = 1;
    bool useTiles = true;
    std::vector<std::vector<int>> tiles;
    std::vector<int> all;
    ~port_ca() { port_bvh_free(tree); }
};

/* makeContactTriangleInfos (SdfBuilder.cpp:155-184) and
 * buildContactTileIndex (SdfBuilder.cpp:202-243). */
port_ca* port_ca_prepare(const double* verts, int nv, const int* tris, int nt,
                         const double* cornerNormals, const port_grid_spec* spec, int tileDim,
                         int useTiles, double influenceRadius)
{
    port_ca* c = new port_ca();
    c->spec = *spec;
    c->tree = port_bvh_build(verts, nv, tris, nt);
    c->tris.resize((size_t)nt);
    for (int t = 0; t < nt; ++t)
    {
        ca_tri& T = c->tris[(size_t)t];
        for (int a = 0; a < 3; ++a)
        {
            T.a[a] = verts[3 * tris[3 * t] + a];
            T.b[a] = verts[3 * tris[3 * t + 1] + a];
            T.c[a] = verts[3 * tris[3 * t + 2] + a];
        }
        for (int v = 0; v < 3; ++v)
            for (int a = 0; a < 3; ++a) T.cn[v][a] = cornerNormals[9 * t + 3 * v + a];
        double e0[3], e1[3], cr[3];
        sub3(T.b, T.a, e0);
        sub3(T.c, T.a, e1);
        cross3(e0, e1, cr);
        normalized_or(cr, kUnitX, T.fn);
        for (int a = 0; a < 3; ++a)
        {
            double mn = T.b[a] < T.a[a] ? T.b[a] : T.a[a];
            mn = T.c[a] < mn ? T.c[a] : mn;
            double mx = T.a[a] < T.b[a] ? T.b[a] : T.a[a];
            mx = mx < T.c[a] ? T.c[a] : mx;
            T.lo[a] = mn;
            T.hi[a] = mx;
        }
    }
    c->all.resize((size_t)nt);
    for (int t = 0; t < nt; ++t) c->all[(size_t)t] = t;
    c->useTiles = useTiles != 0;
    if (!c->useTiles) return c;
    c->tileDim = std::max(1, tileDim);
    c->tnx = (spec->shape[0] + c->tileDim - 1) / c->tileDim;
    c->tny = (spec->shape[1] + c->tileDim - 1) / c->tileDim;
    c->tnz = (spec->shape[2] + c->tileDim - 1) / c->tileDim;
    c->tiles.assign((size_t)c->tnx * c->tny * c->tnz, std::vector<int>());
    const double h = std::max(spec->voxel[0], std::max(spec->voxel[1], spec->voxel[2]));
    const double tileRadius = 0.5 * sqrt(3.0) * (double)c->tileDim * h;
    const double expansion = std::max(0.0, influenceRadius) + tileRadius + h;
    for (int t = 0; t < nt; ++t)
    {
        const ca_tri& T = c->tris[(size_t)t];
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a)
        {
            const double l = T.lo[a] - expansion, u = T.hi[a] + expansion;
            int i0 = (int)floor((l - spec->bmin[a]) / spec->voxel[a] - 0.5);
            int i1 = (int)ceil((u - spec->bmin[a]) / spec->voxel[a] - 0.5);
            i0 = std::max(0, std::min(spec->shape[a] - 1, i0));
            i1 = std::max(0, std::min(spec->shape[a] - 1, i1));
            lo[a] = i0 / c->tileDim;
            hi[a] = i1 / c->tileDim;
        }
        for (int tk = lo[2]; tk <= hi[2]; ++tk)
            for (int tj = lo[1]; tj <= hi[1]; ++tj)
                for (int ti = lo[0]; ti <= hi[0]; ++ti)
                    c->tiles[(size_t)(ti + c->tnx * (tj + c->tny * tk))].push_back(t);
    }
    return c;
}

void port_ca_free(port_ca* c) { delete c; }

static const std::vector<int>& ca_list(const port_ca* c, int i, int j, int k)
{
    if (!c->useTiles) return c->all;
    static const std::vector<int> empty;
    if (c->tiles.empty()) return empty;
    const int ti = std::max(0, std::min(c->tnx - 1, i / c->tileDim));
    const int tj = std::max(0, std::min(c->tny - 1, j / c->tileDim));
    const int tk = std::max(0, std::min(c->tnz - 1, k / c->tileDim));
    return c->tiles[(size_t)(ti + c->tnx * (tj + c->tny * tk))];
}

/* buildContactCandidatesForPoint (SdfBuilder.cpp:268-343) */
static void ca_point(const port_ca* c, const double* p, const std::vector<int>& ids, double tol,
                     double cosMerge, int maxCand, std::vector<ca_cand>& merged)
{
    const int nt = (int)c->tris.size();
    double minDistance = DBL_MAX;
    for (int t : ids)
    {
        if (t < 0 || t >= nt) continue;
        ca_cand cc;
        make_candidate(p, c->tris[(size_t)t], cc);
        minDistance = std::min(minDistance, cc.dist);
    }
    int fallback = -1;
    if (!std::isfinite(minDistance))
    {
        nearest_t nb;
        nearest(c->tree, p, &nb);
        fallback = nb.tri;
        minDistance = nb.tri >= 0 ? sqrt(nb.sq) : DBL_MAX;
    }
    merged.clear();
    const double allowed = minDistance + tol;
    auto tryTri = [&](int t) {
        if (t < 0 || t >= nt) return;
        ca_cand cc;
        make_candidate(p, c->tris[(size_t)t], cc);
        if (cc.dist <= allowed) merge_candidate(merged, cc, cosMerge);
    };
    if (ids.empty())
        tryTri(fallback);
    else
        for (int t : ids) tryTri(t);
    if (merged.empty())
    {
        if (fallback < 0)
        {
            nearest_t nb;
            nearest(c->tree, p, &nb);
            fallback = nb.tri;
        }
        tryTri(fallback);
    }
    std::sort(merged.begin(), merged.end(),
              [](const ca_cand& a, const ca_cand& b) { return fabs(a.phi) < fabs(b.phi); });
    if ((int)merged.size() > maxCand) merged.resize((size_t)maxCand);
}

/* Dense contact-aware fill (SdfBuilder.cpp:472-528): per voxel x-fastest,
 * count[N], cphi[N*s], cnormal[N*s*3], cbranch[N*s] (s = stride), and the
 * primary candidate as phi0[N], n0[N*3], w0[N*3] (left at 0 / UnitX / 0
 * where the voxel has none). */
void port_ca_dense(const port_ca* c, int stride, double tol, double cosMerge, uint8_t* count,
                   double* cphi, double* cn, int* cbr, double* phi0, double* n0, double* w0)
{
    const port_grid_spec* s = &c->spec;
    const int64_t N = (int64_t)s->shape[0] * s->shape[1] * s->shape[2];
#pragma omp parallel for schedule(dynamic, 128)
    for (int64_t idx = 0; idx < N; ++idx)
    {
        const int i = (int)(idx % s->shape[0]);
        const int j = (int)((idx / s->shape[0]) % s->shape[1]);
        const int k = (int)(idx / ((int64_t)s->shape[0] * s->shape[1]));
        double ctr[3];
        center_from_index(s, i, j, k, ctr);
        std::vector<ca_cand> m;
        ca_point(c, ctr, ca_list(c, i, j, k), tol, cosMerge, stride, m);
        const int cnt = std::min((int)m.size(), stride);
        count[idx] = (uint8_t)cnt;
        phi0[idx] = 0.0;
        n0[3 * idx] = 1.0;
        n0[3 * idx + 1] = n0[3 * idx + 2] = 0.0;
        w0[3 * idx] = w0[3 * idx + 1] = w0[3 * idx + 2] = 0.0;
        if (cnt > 0)
        {
            phi0[idx] = m[0].phi;
            memcpy(n0 + 3 * idx, m[0].n, 3 * sizeof(double));
            memcpy(w0 + 3 * idx, m[0].w, 3 * sizeof(double));
        }
        for (int q = 0; q < stride; ++q)
        {
            const int64_t o = idx * stride + q;
            if (q < cnt)
            {
                cphi[o] = m[(size_t)q].phi;
                memcpy(cn + 3 * o, m[(size_t)q].n, 3 * sizeof(double));
                cbr[o] = m[(size_t)q].branch;
            }
            else
            {
                cphi[o] = 0.0;
                cn[3 * o] = 1.0;
                cn[3 * o + 1] = cn[3 * o + 2] = 0.0;
                cbr[o] = -1;
            }
        }
    }
}

/* Sparse contact-aware block selection (SdfBuilder.cpp:593-646): with tiles,
 * a block is active iff a tile it overlaps lists a triangle; without, the
 * nearest-triangle distance from the block centre against activation +
 * block radius.  active[] over all blocks (bi fastest); returns the count. */
int port_ca_sparse_activate(const port_ca* c, int bd, double activation, uint8_t* active)
{
    const port_grid_spec* s = &c->spec;
    const int nbx = (s->shape[0] + bd - 1) / bd, nby = (s->shape[1] + bd - 1) / bd,
              nbz = (s->shape[2] + bd - 1) / bd;
    const int total = nbx * nby * nbz;
    const double h = std::max(s->voxel[0], std::max(s->voxel[1], s->voxel[2]));
    int count = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : count)
    for (int bl = 0; bl < total; ++bl)
    {
        const int bi = bl % nbx, bj = (bl / nbx) % nby, bk = bl / (nbx * nby);
        bool act = false;
        if (c->useTiles && !c->tiles.empty())
        {
            const int i0 = bi * bd, j0 = bj * bd, k0 = bk * bd;
            const int i1 = std::min(i0 + bd - 1, s->shape[0] - 1);
            const int j1 = std::min(j0 + bd - 1, s->shape[1] - 1);
            const int k1 = std::min(k0 + bd - 1, s->shape[2] - 1);
            for (int tk = k0 / c->tileDim; tk <= k1 / c->tileDim && !act; ++tk)
                for (int tj = j0 / c->tileDim; tj <= j1 / c->tileDim && !act; ++tj)
                    for (int ti = i0 / c->tileDim; ti <= i1 / c->tileDim; ++ti)
                        if (!c->tiles[(size_t)(ti + c->tnx * (tj + c->tny * tk))].empty())
                        {
                            act = true;
                            break;
                        }
        }
        else
        {
            const int i0 = bi * bd, j0 = bj * bd, k0 = bk * bd;
            const int i1 = std::min(i0 + bd, s->shape[0]), j1 = std::min(j0 + bd, s->shape[1]),
                      k1 = std::min(k0 + bd, s->shape[2]);
            const double ctr[3] = {s->bmin[0] + s->voxel[0] * (0.5 * (double)(i0 + i1)),
                                   s->bmin[1] + s->voxel[1] * (0.5 * (double)(j0 + j1)),
                                   s->bmin[2] + s->voxel[2] * (0.5 * (double)(k0 + k1))};
            nearest_t nb;
            nearest(c->tree, ctr, &nb);
            const double dist = nb.tri >= 0 ? sqrt(nb.sq) : DBL_MAX;
            const double blockRadius = 0.5 * sqrt(3.0) * (double)bd * h;
            act = dist <= activation + blockRadius;
        }
        active[bl] = act ? 1 : 0;
        count += act ? 1 : 0;
    }
    return count;
}

/* Sparse contact-aware brick fill (SdfBuilder.cpp:680-770), FP32 storage:
 * phi (B,V), normal (B,V,3), count (B,V), cphi (B,V,s), cn (B,V,s,3),
 * cbr (B,V,s). */
void port_ca_sparse_fill(const port_ca* c, int bd, int nblocks, const int* ijk, int stride,
                         double tol, double cosMerge, float* phi, float* normal, uint8_t* count,
                         float* cphi, float* cn, int* cbr)
{
    const port_grid_spec* s = &c->spec;
    const int V = bd * bd * bd;
#pragma omp parallel for schedule(dynamic, 1)
    for (int b = 0; b < nblocks; ++b)
    {
        std::vector<ca_cand> m;
        for (int local = 0; local < V; ++local)
        {
            const int lx = local % bd, ly = (local / bd) % bd, lz = local / (bd * bd);
            const int i = ijk[3 * b] * bd + lx, j = ijk[3 * b + 1] * bd + ly, k = ijk[3 * b + 2] * bd + lz;
            const int64_t v = (int64_t)b * V + local;
            for (int q = 0; q < stride; ++q)
            {
                cphi[v * stride + q] = 0.f;
                cn[3 * (v * stride + q)] = cn[3 * (v * stride + q) + 1] = cn[3 * (v * stride + q) + 2] = 0.f;
                cbr[v * stride + q] = -1;
            }
            phi[v] = 0.f;
            normal[3 * v] = 1.f;
            normal[3 * v + 1] = normal[3 * v + 2] = 0.f;
            count[v] = 0;
            if (!in_bounds(s, i, j, k)) continue;
            double ctr[3];
            center_from_index(s, i, j, k, ctr);
            ca_point(c, ctr, ca_list(c, i, j, k), tol, cosMerge, stride, m);
            const int cnt = std::min((int)m.size(), stride);
            count[v] = (uint8_t)cnt;
            if (cnt > 0)
            {
                phi[v] = (float)m[0].phi;
                for (int a = 0; a < 3; ++a) normal[3 * v + a] = (float)m[0].n[a];
            }
            for (int q = 0; q < cnt; ++q)
            {
                const int64_t o = v * stride + q;
                cphi[o] = (float)m[(size_t)q].phi;
                for (int a = 0; a < 3; ++a) cn[3 * o + a] = (float)m[(size_t)q].n[a];
                cbr[o] = m[(size_t)q].branch;
            }
        }
    }
}

/* queryFast ContactAware branch (SdfOracle.cpp:296-423) for one point given
 * its voxel's candidates (count > 0): gap, normal, witness of the candidate
 * with the smallest |gap| (first on ties), and every candidate's (gap,
 * normal, witness, branch). */
static void ca_eval(const double* p, const double* ctr, int cnt, const double* cphi,
                    const double* cn, const int* cbr, double* gap, double* nrm, double* wit,
                    double* kgap, double* kn, double* kw, int* kb)
{
    double dx[3];
    sub3(p, ctr, dx);
    int sel = 0;
    double best = DBL_MAX;
    for (int q = 0; q < cnt; ++q)
    {
        double n[3] = {cn[3 * q], cn[3 * q + 1], cn[3 * q + 2]};
        const double l = norm3(n);
        if (l > 1.0e-15)
            for (int a = 0; a < 3; ++a) n[a] /= l;
        else
        {
            n[0] = 1.0;
            n[1] = n[2] = 0.0;
        }
        const double g = cphi[q] + dot3(n, dx);
        kgap[q] = g;
        for (int a = 0; a < 3; ++a)
        {
            kn[3 * q + a] = n[a];
            kw[3 * q + a] = p[a] - g * n[a];
        }
        kb[q] = cbr[q];
        if (fabs(g) < best)
        {
            best = fabs(g);
            sel = q;
        }
    }
    *gap = kgap[sel];
    for (int a = 0; a < 3; ++a)
    {
        nrm[a] = kn[3 * sel + a];
        wit[a] = kw[3 * sel + a];
    }
}

/* Dense ContactAware queries.  Per point: valid, gap, normal[3], witness[3],
 * ncand (0 where the voxel has no candidate: the point then takes the
 * FirstOrder query, done by the caller), and up to 8 candidates
 * (kgap[n*8], kn[n*24], kw[n*24], kb[n*8]). */
void port_ca_query_dense(const port_grid_spec* s, int stride, const uint8_t* count,
                         const double* cphi, const double* cn, const int* cbr, const double* pts,
                         int64_t n, uint8_t* valid, double* gap, double* nrm, double* wit,
                         int* ncand, double* kgap, double* kn, double* kw, int* kb)
{
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; ++q)
    {
        const double* p = pts + 3 * q;
        int ijk[3];
        for (int a = 0; a < 3; ++a) ijk[a] = (int)round((p[a] - s->bmin[a]) / s->voxel[a] - 0.5);
        valid[q] = 0;
        ncand[q] = 0;
        if (!in_bounds(s, ijk[0], ijk[1], ijk[2])) continue;
        const int64_t v = ijk[0] + (int64_t)s->shape[0] * (ijk[1] + (int64_t)s->shape[1] * ijk[2]);
        const int cnt = std::min((int)count[v], stride);
        valid[q] = 1;
        if (cnt <= 0) continue;
        const int kc = std::min(cnt, 8);
        double ctr[3];
        center_from_index(s, ijk[0], ijk[1], ijk[2], ctr);
        ncand[q] = kc;
        ca_eval(p, ctr, kc, cphi + v * stride, cn + 3 * v * stride, cbr + v * stride, gap + q,
                nrm + 3 * q, wit + 3 * q, kgap + 8 * q, kn + 24 * q, kw + 24 * q, kb + 8 * q);
    }
}

/* Sparse ContactAware queries (FP32 candidate storage widened to FP64). */
void port_ca_query_sparse(const port_grid_spec* s, int bd, int nblocks, const int* ijk,
                          int stride, const uint8_t* count, const float* cphi, const float* cn,
                          const int* cbr, const double* pts, int64_t n, uint8_t* valid,
                          double* gap, double* nrm, double* wit, int* ncand, double* kgap,
                          double* kn, double* kw, int* kb)
{
    sparse_index x;
    sparse_index_init(&x, s, bd, nblocks, ijk);
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < n; ++q)
    {
        const double* p = pts + 3 * q;
        int c3[3];
        for (int a = 0; a < 3; ++a) c3[a] = (int)round((p[a] - s->bmin[a]) / s->voxel[a] - 0.5);
        valid[q] = 0;
        ncand[q] = 0;
        if (!in_bounds(s, c3[0], c3[1], c3[2])) continue;
        const int64_t v = sparse_voxel(&x, c3[0], c3[1], c3[2]);
        if (v < 0) continue;
        const int cnt = std::min((int)count[v], stride);
        valid[q] = 1;
        if (cnt <= 0) continue;
        const int kc = std::min(cnt, 8);
        double ph[8], nn[24];
        for (int k = 0; k < kc; ++k)
        {
            ph[k] = (double)cphi[v * stride + k];
            for (int a = 0; a < 3; ++a) nn[3 * k + a] = (double)cn[3 * (v * stride + k) + a];
        }
        double ctr[3];
        center_from_index(s, c3[0], c3[1], c3[2], ctr);
        ncand[q] = kc;
        ca_eval(p, ctr, kc, ph, nn, cbr + v * stride, gap + q, nrm + 3 * q, wit + 3 * q,
                kgap + 8 * q, kn + 24 * q, kw + 24 * q, kb + 8 * q);
    }
    free(x.table);
}
