/*
 * sdfo_port.h -- CPU restatement of the SdfOracle hot path (oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA kernels are compared
 * against; the product never links or calls it.  Every function restates the
 * reference algorithm in plain C with the reference's FP64 operation order
 * (compiled with -ffp-contract=off), citing the reference file:line it
 * follows.  Parity of this restatement with the reference itself is pinned by
 * tests against golden vectors produced by the reference sources
 * (oracle/_ref, tests/golden/make_golden.py).
 *
 * The triangle tree is the reference's (median split with std::nth_element,
 * leaves of 8, near-first depth-first search), so exact ties between
 * equidistant triangles resolve to the same triangle as in the reference:
 * the face-normal sign fallback for points the parity ray misses depends on
 * that choice.
 */
#ifndef SDFO_PORT_H
#define SDFO_PORT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
    double bmin[3];
    double bmax[3];
    double voxel[3];
    int shape[3];
} port_grid_spec;

enum
{
    PORT_FIRST_ORDER = 0,
    PORT_SECOND_ORDER = 1,
    PORT_TRILINEAR = 2,
    PORT_TRICUBIC = 3
};

/* SdfBuilder::setupGrid (SdfBuilder.cpp:994-1035) + snapToStandardResolution
 * (GridSpec.h:65-74). */
void port_setup_grid(const double* verts, int nv, double padding, double voxelSize,
                     int targetResolution, int maxResolution, port_grid_spec* out);
int port_snap_resolution(int n, int maxRes);

typedef struct port_bvh port_bvh;
port_bvh* port_bvh_build(const double* verts, int nv, const int* tris, int nt);
void port_bvh_free(port_bvh* b);

/* KdTree::findSignedNearest (KdTree.h:143-165) for n points: signed distance,
 * closest point, face normal of the chosen triangle, triangle index and the
 * ray-parity hit count (countRayIntersections, KdTree.h:398-441). */
void port_signed_nearest(const port_bvh* b, const double* pts, int64_t n, double* sd,
                         double* cp, double* fn, int* tri, int* hits);
/* Unsigned nearest distance only (used for sparse block activation). */
void port_nearest_distance(const port_bvh* b, const double* pts, int64_t n, double* dist);
/* The findSignedNearest traversals of n points, counted (serial): counts[0]
 * nodes entered past the nearest search's cut, [1] closest-point tests,
 * [2] ray-box tests, [3] ray-triangle tests. */
void port_traversal_counts(const port_bvh* b, const double* pts, int64_t n, int64_t* counts);

/* Dense build: computeSdfAndNormals (SdfBuilder.cpp:1039-1101) then
 * estimateHessian (SdfBuilder.cpp:1105-1152).  Arrays are x-fastest,
 * normal/witness (N,3), hess6 (N,6) = xx,xy,xz,yy,yz,zz.  Any output may be
 * NULL except phi and normal. */
void port_build_dense(const port_bvh* b, const port_grid_spec* spec, double* phi,
                      double* normal, double* hess6, double* witness);
void port_dense_hessian(const port_grid_spec* spec, const double* normal, double* hess6);

/* Sparse narrow-band build (SdfBuilder.cpp:823-983).  activate: flags for all
 * nbx*nby*nbz blocks in linear (bi fastest) order, returns active count.
 * fill: per-block FP32 phi (B,V) and normal (B,V,3) for the given block list.
 * hessian: estimateSparseHessian (SdfBuilder.cpp:1154-1225). */
int port_sparse_activate(const port_bvh* b, const port_grid_spec* spec, int blockDim,
                         int haloVoxels, double bandDistance, uint8_t* active);
void port_sparse_fill(const port_bvh* b, const port_grid_spec* spec, int blockDim, int nblocks,
                      const int* ijk, float* phi, float* normal);
void port_sparse_hessian(const port_grid_spec* spec, int blockDim, int nblocks, const int* ijk,
                         const float* normal, float* hess6);

/* Queries.  Outputs (any may be NULL): gap[n], grad[n*3] (raw gradient of the
 * interpolant; for FirstOrder/SecondOrder the normal it returns), unit[n*3]
 * (the reference's gapNormal incl. its UnitX fallback), witness[n*3],
 * valid[n], hess[n*9] (d grad / d p of the interpolant, row-major).
 * Dense: SdfOracle.cpp:448-596, 932-1092.  Sparse: SdfOracle.cpp:600-851. */
void port_query_dense(const port_grid_spec* spec, const double* phi, const double* normal,
                      const double* hess6, int mode, const double* pts, int64_t n, double* gap,
                      double* grad, double* unit, double* witness, uint8_t* valid, double* hess);
void port_query_sparse(const port_grid_spec* spec, int blockDim, int nblocks, const int* ijk,
                       const float* phi, const float* normal, const float* hess6, int mode,
                       const double* pts, int64_t n, double* gap, double* grad, double* unit,
                       double* witness, uint8_t* valid, double* hess);

/* Contact-aware builds (SdfBuilder.cpp:27-359 helpers, 416-821) and the
 * ContactAware branch of queryFast (SdfOracle.cpp:269-431).  prepare: the
 * triangle records (corner normals (nt,3,3)), the reference tree for the
 * nearest-triangle fallback and, with useTiles, the tile index (tileDim^3
 * voxel tiles, triangles whose bounds grown by influenceRadius + tile radius
 * + h overlap the tile, in triangle order). */
typedef struct port_ca port_ca;
port_ca* port_ca_prepare(const double* verts, int nv, const int* tris, int nt,
                         const double* cornerNormals, const port_grid_spec* spec, int tileDim,
                         int useTiles, double influenceRadius);
void port_ca_free(port_ca* c);
void port_ca_dense(const port_ca* c, int stride, double tol, double cosMerge, uint8_t* count,
                   double* cphi, double* cn, int* cbr, double* phi0, double* n0, double* w0);
int port_ca_sparse_activate(const port_ca* c, int bd, double activation, uint8_t* active);
void port_ca_sparse_fill(const port_ca* c, int bd, int nblocks, const int* ijk, int stride,
                         double tol, double cosMerge, float* phi, float* normal, uint8_t* count,
                         float* cphi, float* cn, int* cbr);
void port_ca_query_dense(const port_grid_spec* s, int stride, const uint8_t* count,
                         const double* cphi, const double* cn, const int* cbr, const double* pts,
                         int64_t n, uint8_t* valid, double* gap, double* nrm, double* wit,
                         int* ncand, double* kgap, double* kn, double* kw, int* kb);
void port_ca_query_sparse(const port_grid_spec* s, int bd, int nblocks, const int* ijk,
                          int stride, const uint8_t* count, const float* cphi, const float* cn,
                          const int* cbr, const double* pts, int64_t n, uint8_t* valid,
                          double* gap, double* nrm, double* wit, int* ncand, double* kgap,
                          double* kn, double* kw, int* kb);

void port_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
