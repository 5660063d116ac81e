/*
 * sdfo.h -- C ABI of libsdfo_cuda.so, the B200 (sm_100a) implementation of
 * the SdfOracle hot path: SDF construction from a triangle mesh (dense and
 * sparse narrow-band), batched SDF queries with their backward, and the fused
 * per-quadrature-point penalty contact with its 6-DoF pose Jacobian.
 *
 * Conventions
 *  - Plain C: no C++ types, no exceptions cross this boundary.  Every
 *    function returns an int status: SDFO_OK (0) or a negative SDFO_ERR_*;
 *    sdfo_last_error() returns the message of the calling thread's last error.
 *  - Pointers named d_* are device pointers (CUDA global memory, e.g. a torch
 *    tensor's data_ptr()); pointers named h_* are host pointers.  `stream` is
 *    a cudaStream_t passed as void* (NULL = legacy default stream).  Calls
 *    taking d_* buffers are asynchronous on `stream` unless stated.
 *  - Buffers are owned by the caller.  The library owns only the storage
 *    behind an sdfo_grid handle.  A handle is immutable after creation, so
 *    concurrent queries on different streams are safe.
 *  - Grid index convention (reference GridSpec, GridSpec.h:17-60): voxel
 *    centre = bmin + voxel * (ijk + 0.5); linear index i + nx*(j + ny*k).
 *
 * The reference (W-Moorer/sdf-contact-module) has no FFI; each entry point
 * below names the reference interface whose behaviour it reproduces.
 */
#ifndef SDFO_H
#define SDFO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SDFO_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
#define SDFO_OK 0
#define SDFO_ERR_INVALID_ARGUMENT (-1) /* bad pointer, size, mode or params */
#define SDFO_ERR_CUDA (-2)             /* a CUDA runtime call failed */
#define SDFO_ERR_OUT_OF_MEMORY (-3)
#define SDFO_ERR_EMPTY_MESH (-4)       /* "Empty mesh provided to SdfBuilder" */
#define SDFO_ERR_DEVICE_STATUS (-5)    /* a kernel reported a failure (see message) */
#define SDFO_ERR_UNSUPPORTED (-6)      /* mode/layout combination not provided */
#define SDFO_ERR_NO_DEVICE (-7)        /* no CUDA device / not an sm_100 device */
#define SDFO_ERR_IO (-8)               /* a file cannot be opened, read or written, or
                                          is not an SDFO 0.1.0 file of the asked layout */

/* ---- enums --------------------------------------------------------------- */
/* QueryMode (SdfOracle.h:11-18). */
#define SDFO_FIRST_ORDER 0
#define SDFO_SECOND_ORDER 1
#define SDFO_TRILINEAR 2
#define SDFO_TRICUBIC 3
#define SDFO_CONTACT_AWARE 4

/* Storage layouts, numbered as the SDFO 0.1.0 header's layout field
 * (SdfIO.cpp:30-33). */
#define SDFO_LAYOUT_DENSE 1
#define SDFO_LAYOUT_SPARSE 2

/* Device storage precision of the query payload. */
#define SDFO_STORAGE_FP32 0
#define SDFO_STORAGE_FP16 1 /* sparse only: per-brick affine phi + fp16 normal */

/* Triangle acceleration structure used by the builders. */
#define SDFO_BVH_REFERENCE 0 /* the reference's median-split tree (host-built),
                                traversed on the device in its order: results
                                identical to the reference incl. exact ties */
#define SDFO_BVH_LBVH 1      /* device-built linear BVH: fastest build; exactly
                                equidistant triangles resolve to the lowest
                                index, so witness/normal at such ties and the
                                face-normal sign fallback may differ */

/* Inside/outside sign rule of the builders. */
#define SDFO_SIGN_RAY_PARITY 0   /* the reference's: parity of the hits of one
                                    fixed ray, the nearest triangle's face
                                    normal when it hits nothing
                                    (KdTree.h:143-165, 330-441) */
#define SDFO_SIGN_PSEUDONORMAL 1 /* angle-weighted pseudo-normal of the
                                    closest point's feature (vertex, edge or
                                    face); needs a closed, consistently
                                    oriented mesh; no parity ray; the sign
                                    does not depend on which of several
                                    equidistant triangles is kept */

/* Point precision for query inputs. */
#define SDFO_POINTS_F32 0
#define SDFO_POINTS_F64 1

typedef struct sdfo_grid sdfo_grid;

/* GridSpec (GridSpec.h:17-27) plus the sparse header fields of
 * SparseSdfData (SdfData.h:154-163). */
typedef struct
{
    double bmin[3];
    double bmax[3];
    double voxel[3];
    int32_t shape[3];       /* nx, ny, nz */
    int32_t layout;         /* SDFO_LAYOUT_* */
    int32_t storage;        /* SDFO_STORAGE_* */
    int32_t has_hessian;
    int32_t block_dim;      /* sparse */
    int32_t halo_voxels;    /* sparse */
    int32_t block_count;    /* sparse: number of stored blocks */
    int32_t candidate_stride; /* contact-aware candidate slots per voxel, 0 = none */
    double band_distance;   /* sparse */
} sdfo_grid_info;

/* BuilderParams (SdfBuilder.h:24-31); the log callback stays on the host. */
typedef struct
{
    double padding;            /* fraction of the bbox diagonal, default 0.1 */
    double voxel_size;         /* 0 = longest padded side / target_resolution */
    int32_t target_resolution; /* default 128 */
    int32_t max_resolution;    /* default 512 */
} sdfo_build_params;

/* SparseBuilderParams (SdfBuilder.h:33-40). */
typedef struct
{
    sdfo_build_params base;
    int32_t block_dim;     /* default 8 */
    int32_t halo_voxels;   /* default 2 */
    int32_t band_voxels;   /* default 8 */
    int32_t store_hessian; /* default 1 */
    double band_distance;  /* 0 = band_voxels * voxel */
} sdfo_sparse_build_params;

/* ContactAwareBuilderParams (SdfBuilder.h:42-55). */
typedef struct
{
    sdfo_build_params base;
    int32_t max_candidates;            /* default 4; at most 8 are stored */
    int32_t tile_dim;                  /* default 8 */
    int32_t use_tile_acceleration;     /* default 1 */
    int32_t store_hessian;             /* default 1 */
    double feature_distance_tolerance; /* 0 = 1.5 * voxel */
    double normal_merge_angle_degrees; /* default 5 */
    int32_t sparse;                    /* default 0 */
    int32_t block_dim;                 /* default 8 */
    int32_t halo_voxels;               /* default 2 */
    int32_t band_voxels;               /* default 8 */
    double band_distance;              /* 0 = band_voxels * voxel */
} sdfo_contact_aware_params;

/* Body state for contact: position r, rotation R (row-major 3x3, body to
 * world), linear velocity v and angular velocity w (world frame). */
typedef struct
{
    double r[3];
    double R[9];
    double v[3];
    double w[3];
} sdfo_body_state;

/* ContactPair fields used by SDFContactEngine.evaluate
 * (prototype/src/ir/contact.py:1-18, contacts_sdf.py:296-302). */
typedef struct
{
    double stiffness;           /* k_n */
    double order;               /* k_order (n in k * delta^n) */
    double damping;             /* c_n, quadrature_settings['damping'] */
    double friction;            /* mu */
    double regularizer;         /* quadrature_settings['regularizer'] */
    double activation_distance; /* read but unused by the reference law */
} sdfo_contact_params;

/* ContactMeasure (contacts_sdf.py:8-17) of one pose, from measure_pair
 * (contacts_sdf.py:171-214): the minimum gap over the in-grid quadrature
 * points the broad phase keeps (+inf when there is none), its penetration
 * max(0, -gap), the normal relative velocity at that point, the point's
 * index in the broad phase's point list (-1 when none), and the counts of
 * in-grid points with gap < 0 and of in-grid points. */
typedef struct
{
    double gap;
    double penetration;
    double normal_velocity;
    int32_t min_point_index;
    int32_t active_count;
    int32_t valid_count;
    int32_t reserved0;
} sdfo_contact_measure;

/* Build statistics of the last build on a handle: setup_ms = host grid
 * setup and the grid's device allocations, bvh_ms = acceleration structure,
 * fill_ms = distance / sign fill, hessian_ms = Hessian and query layouts. */
typedef struct
{
    double setup_ms, bvh_ms, fill_ms, hessian_ms, total_ms;
    int64_t voxels_filled;    /* voxels whose distance was computed */
    int64_t candidate_blocks; /* sparse: blocks tested for activation */
    int32_t triangles;
    int32_t bvh_nodes;
} sdfo_build_stats;

/* Raw device views of a grid (for interop, e.g. torch autograd on the
 * payload).  Dense: phin = float4[nx*ny*nz] {phi, nx, ny, nz}.  Sparse:
 * phin = float4[block_count * block_dim^3], table = int32[nbx*nby*nbz]
 * (block slot or -1), block_ijk = int32[block_count*3]. */
typedef struct
{
    void* phin;
    void* hessian6; /* float[6] per stored voxel, or NULL */
    void* table;
    void* block_ijk;
    int64_t stored_voxels;
    int32_t table_dims[3];
    int32_t reserved0;
} sdfo_device_views;

/* ---- library ------------------------------------------------------------ */
const char* sdfo_version(void);
int sdfo_abi_version(void);
/* Copies the calling thread's last error message (NUL-terminated). */
int sdfo_last_error(char* buf, size_t len);
/* Checks that device `device` is usable (compute capability 10.x). */
int sdfo_device_check(int device);

/* Device memory the library frees (grids, build temporaries) is kept for
 * reuse by later requests of the same size class, up to `limit` bytes per
 * device (default 1 GiB).  A free still synchronises the device first, as
 * cudaFree does.  limit < 0 leaves the limit as it is; 0 releases every
 * cached block of the current device and turns the cache off.  *held (may
 * be NULL) receives the bytes now cached on the current device. */
int sdfo_device_cache(int64_t limit, int64_t* held);

/* Status word the kernels with bounded waits set instead of hanging (bit 0:
 * a bulk-copy wait of the saved backward's pipeline ran out; bit 1: a wait
 * of the pipelined dense query kernel ran out -- with the default
 * sdfo_tuning.query_walk only the dense linearising forward runs that
 * kernel); synchronous read, cleared when `clear` != 0.  0 in normal
 * operation.  The synchronous host
 * entry points (sdfo_query_host, sdfo_query_host_static) read bit 1 in
 * stream order themselves and return SDFO_ERR_DEVICE_STATUS (clearing it)
 * when it is set; after the asynchronous calls (sdfo_query,
 * sdfo_query_linearize, sdfo_query_backward_saved on device buffers) the
 * caller checks this word once the stream has finished. */
int sdfo_device_status(uint32_t* flags, int32_t clear);

/* Test-only (no reference counterpart): shortens the main-loop wait of the
 * two bulk-copy pipelines (k_query_pipe, k_backward_saved_bulk) to
 * `wait_limit` try-wait iterations (0 = the built-in limit) and, when
 * `withhold_first_tile` != 0, makes every CTA skip the bulk load of its first
 * tile so that the wait for it runs out.  The kernel then sets its status bit,
 * waits for the loads it did issue and returns; nothing faults or hangs.
 * Process-wide; sdfo_debug_wait_test(0, 0) restores normal operation. */
int sdfo_debug_wait_test(uint32_t wait_limit, int32_t withhold_first_tile);

/* Process-wide tuning knobs (no reference counterpart; the reference has no
 * device code to tune).  Zero selects the default of a field.  The autotuner
 * (sdfo/tune.py) times candidates on the caller's data and stores its picks
 * keyed by GPU and workload shape. */
typedef struct
{
    int32_t host_chunk_queries; /* sdfo_query_host with pinned buffers: queries of the
                                   first pipelined chunk (rounded up to 256;
                                   default 32768); n <= this: no pipelining */
    int32_t fill_ctas_per_sm;   /* batched brick fill: CTAs per SM (0 = as many as fit) */
    int32_t fill_tile_log2_x;   /* dense fill: voxel tile of a 256-thread CTA is */
    int32_t fill_tile_log2_y;   /* 2^x by 2^y by 256/2^(x+y), x fastest (0 = 3: 8x8x4) */
    int32_t lbvh_traversal;     /* SDFO_BVH_LBVH traversals: 1 = per-thread stack,
                                   2 = stackless (parent links); 0 = default (2);
                                   same results and work either way */
    int32_t host_chunk_growth_pct; /* each next pipelined chunk is this percent of
                                      the previous (100..400; 0 = default 130) */
    int32_t host_io_mode;       /* sdfo_query_host with pinned buffers: 1 = staged in
                                   device memory, copied in and out per chunk;
                                   2 = points copied in per chunk, results written
                                   by the query straight into the caller's buffers;
                                   3 = one query launch reads the points from and
                                   writes the results to the caller's buffers (both
                                   mapped into the device), no staging; modes 2 and
                                   3 fall back to 1 for unmapped buffers; 0 = default
                                   (3) */
    int32_t triangle_cull;      /* reference-order tree: 1 = a conservative FP32
                                   triangle-box test skips closest-point tests that
                                   cannot replace the best (same results), 2 = off;
                                   0 = default (1) */
    int32_t sparse_pair_records; /* sparse FP32 grids with 8^3 bricks created from
                                    now on keep a 32-byte record {voxel, +x
                                    neighbour} per stored voxel (one 256-bit load
                                    per Tricubic row; twice the payload's memory):
                                    0 = when the payload is at most 48 MB (the
                                    records then stay in L2; larger pools gather
                                    from DRAM, where the doubled footprint costs
                                    more), 1 = always, 2 = never */
    int32_t query_walk;         /* Trilinear / Tricubic queries and their
                                   regathering backward for dL/dp (and ContactAware
                                   queries of sparse grids) of FP32 points with
                                   results in device memory: 2 = persistent CTAs
                                   over contiguous tile ranges, next point
                                   prefetched, no CTA barriers (sparse grids: every
                                   output, 18% faster than 1 on the 512^3
                                   icosphere; dense grids: without the Hessian, 13%
                                   faster than the bulk-copy pipeline on the hollow
                                   cylinder); 1 = per-tile kernels (points and
                                   results staged through shared memory, or the
                                   dense bulk-copy pipeline); same results;
                                   0 = default (2) */
} sdfo_tuning;
int sdfo_set_tuning(const sdfo_tuning* t);
int sdfo_get_tuning(sdfo_tuning* t);

void sdfo_build_params_default(sdfo_build_params* p);
void sdfo_sparse_build_params_default(sdfo_sparse_build_params* p);
void sdfo_contact_aware_params_default(sdfo_contact_aware_params* p);

/* Host-only grid setup: SdfBuilder::setupGrid (SdfBuilder.cpp:994-1035) with
 * snapToStandardResolution (GridSpec.h:65-74). */
int sdfo_setup_grid(const double* h_verts, int64_t nv, const sdfo_build_params* p,
                    sdfo_grid_info* out);

/* ---- build (SdfBuilder) --------------------------------------------------- */
/* SdfBuilder::build (SdfBuilder.cpp:364-407, SdfBuilder.h:62-70): dense SDF,
 * normals, witness points and symmetrised Hessian.  h_verts (nv,3) float64,
 * h_tris (nt,3) int32, both host.  Synchronous. */
int sdfo_grid_build_dense(const double* h_verts, int64_t nv, const int32_t* h_tris, int64_t nt,
                          const sdfo_build_params* p, void* stream, sdfo_grid** out);

/* SdfBuilder::buildSparse (SdfBuilder.cpp:823-983, SdfBuilder.h:83-91):
 * narrow-band blocks in (bk, bj, bi) order, FP32 payload.  Synchronous. */
int sdfo_grid_build_sparse(const double* h_verts, int64_t nv, const int32_t* h_tris, int64_t nt,
                           const sdfo_sparse_build_params* p, void* stream, sdfo_grid** out);

/* SdfBuilder::buildContactAware / buildSparseContactAware (p->sparse)
 * (SdfBuilder.cpp:416-821): per voxel up to min(max_candidates, 8)
 * surface-feature candidates {phi, normal, FNV branch id} from the
 * triangles within the nearest distance + tolerance, merged by normal angle
 * and sorted by |phi|; the first is the voxel's phi / n / witness.
 * h_corner_normals (nt, 3, 3) float64: the three corner normals of each
 * triangle (CornerNormalTriangleMesh).  At most 512 merged normal groups per
 * voxel before truncation to max_candidates (more returns
 * SDFO_ERR_UNSUPPORTED).  Synchronous. */
int sdfo_grid_build_contact_aware(const double* h_verts, int64_t nv, const int32_t* h_tris,
                                  int64_t nt, const double* h_corner_normals,
                                  const sdfo_contact_aware_params* p, void* stream,
                                  sdfo_grid** out);

/* One mesh of a batched build: host arrays as for sdfo_grid_build_sparse. */
typedef struct
{
    const double* h_verts; /* (nv, 3) float64 */
    int64_t nv;
    const int32_t* h_tris; /* (nt, 3) int32 */
    int64_t nt;
    sdfo_sparse_build_params params;
} sdfo_mesh_desc;

/* Many sparse builds in one pass (no reference counterpart as a single
 * call; each grid equals SdfBuilder::buildSparse of its mesh and params):
 * the per-mesh trees are built on host threads (or on the device in LBVH
 * mode), then ONE block-activation launch over every mesh's candidate
 * blocks, one scan, ONE persistent brick-fill launch whose CTAs take bricks
 * of any mesh from a shared work counter (meshes of very different sizes
 * load-balance), and one Hessian launch.  All meshes must use the same
 * block_dim.  out[n] receives one handle per mesh; the handles share one
 * device allocation, released with the last of them.  Synchronous. */
int sdfo_grid_build_sparse_batched(const sdfo_mesh_desc* meshes, int32_t n, void* stream,
                                   sdfo_grid** out);
/* CTAs per SM of the persistent brick fill of batched builds (process-wide;
 * 0 = as many as fit, the default) -- a knob of the autotuner. */
int sdfo_set_fill_ctas_per_sm(int32_t ctas);

int sdfo_grid_build_stats(const sdfo_grid* g, sdfo_build_stats* out);

/* Traversal work of the dense fill (no reference counterpart; for
 * profiling): the nearest-triangle searches (KdTree::findNearest) and the
 * parity-ray counts (countRayIntersections) of every voxel of the grid that
 * `p` gives, on the current acceleration structure, run by an instrumented
 * copy of the fill kernel that counts instead of storing.  Synchronous. */
typedef struct
{
    int64_t voxels;
    int64_t nearest_nodes;     /* nodes whose children or triangles were examined */
    int64_t nearest_triangles; /* closest-point tests */
    int64_t ray_nodes;         /* ray-box tests */
    int64_t ray_triangles;     /* ray-triangle tests */
    int64_t nearest_triangles_exact; /* closest-point tests run in FP64: those
                                        not skipped by the conservative FP32
                                        triangle-box cull (reference-order tree) */
} sdfo_traversal_stats;
int sdfo_build_traversal_stats(const double* h_verts, int64_t nv, const int32_t* h_tris, int64_t nt,
                               const sdfo_build_params* p, void* stream, sdfo_traversal_stats* out);

/* Selects the acceleration structure of subsequent builds (process-wide;
 * default SDFO_BVH_REFERENCE).  No reference counterpart: the reference has
 * only its own tree. */
int sdfo_set_bvh_mode(int32_t mode);
int sdfo_get_bvh_mode(void);

/* Selects the sign rule of subsequent builds (process-wide; default
 * SDFO_SIGN_RAY_PARITY, the reference's).  SDFO_SIGN_PSEUDONORMAL has no
 * reference counterpart: distances, closest points and the sparse block set
 * are unchanged; only the sign rule differs.  The per-triangle pseudo-normals
 * are computed on the host at each build (an edge hash map: O(triangles)). */
int sdfo_set_sign_mode(int32_t mode);
int sdfo_get_sign_mode(void);

/* ---- grid from / to host data (SdfData / SparseSdfData, SdfData.h) ------- */
/* SdfOracle(SdfData) (SdfOracle.cpp:154-157): dense FP64 arrays, x-fastest:
 * phi (N), normal (N,3), hessian6 (N,6: xx,xy,xz,yy,yz,zz, may be NULL),
 * witness (N,3, may be NULL).  info supplies bmin/bmax/voxel/shape. */
int sdfo_grid_create_dense(const sdfo_grid_info* info, const double* h_phi,
                           const double* h_normal, const double* h_hessian6,
                           const double* h_witness, void* stream, sdfo_grid** out);
/* SdfOracle(SparseSdfData) (SdfOracle.cpp:159-163): block_count blocks of
 * block_dim^3 voxels: ijk (B,3), phi (B,V), normal (B,V,3), hessian6 (B,V,6)
 * or NULL.  Blocks are kept in the given order. */
int sdfo_grid_create_sparse(const sdfo_grid_info* info, const int32_t* h_block_ijk,
                            const float* h_phi, const float* h_normal, const float* h_hessian6,
                            void* stream, sdfo_grid** out);
/* Re-encodes a sparse FP32 grid as FP16 with a per-brick phi scale/offset
 * (new storage form; the SDFO file format is unchanged). */
int sdfo_grid_to_fp16(const sdfo_grid* src, void* stream, sdfo_grid** out);

/* Export to host in the SdfData / SparseSdfData layouts above.  Dense grids
 * built on the device keep their FP64 build results, so the export is
 * exact; dense grids created from FP32-only data widen to FP64. */
int sdfo_grid_export_dense(const sdfo_grid* g, double* h_phi, double* h_normal,
                           double* h_hessian6, double* h_witness);
int sdfo_grid_export_sparse(const sdfo_grid* g, int32_t* h_block_ijk, float* h_phi,
                            float* h_normal, float* h_hessian6);

/* Copies the grid's FP32 query payload (float4 {phi, n} per stored voxel,
 * dense x-fastest or sparse brick order) into d_dst. */
int sdfo_grid_copy_payload(const sdfo_grid* g, void* d_dst, void* stream);
/* A handle that shares g's structure (spec, block table) but reads its FP32
 * payload from caller-owned device memory d_phin (stored_voxels float4, not
 * copied, not freed).  Used to differentiate w.r.t. the payload held in a
 * framework tensor.  Must be destroyed before g and before d_phin is freed. */
/* Contact-aware candidates of a grid (candidate_stride s > 0), host
 * arrays in stored-voxel order: h_count (N) u8, h_phi (N*s), h_normal
 * (N*s*3), h_branch (N*s) -- SdfData::contactCandidate* (SdfData.h:46-50)
 * and SparseSdfBlock::contactCandidate* (SdfData.h:126-129); sparse values
 * are the stored FP32 widened.  Any output may be NULL. */
int sdfo_grid_export_candidates(const sdfo_grid* g, uint8_t* h_count, double* h_phi,
                                double* h_normal, int32_t* h_branch);
/* Attaches contact-aware candidates (same layout) to a grid made by
 * sdfo_grid_create_dense / _sparse, e.g. from a contact-aware SDFO file;
 * call before the grid is queried.  stride 1..8. */
int sdfo_grid_attach_candidates(sdfo_grid* g, int32_t stride, const uint8_t* h_count,
                                const double* h_phi, const double* h_normal,
                                const int32_t* h_branch);

int sdfo_grid_create_view(const sdfo_grid* g, void* d_phin, sdfo_grid** out);

int sdfo_grid_get_info(const sdfo_grid* g, sdfo_grid_info* out);
int sdfo_grid_device_views(const sdfo_grid* g, sdfo_device_views* out);
int sdfo_grid_destroy(sdfo_grid* g);

/* ---- SDFO 0.1.0 files, device-direct (SdfIO.cpp:93-552) ------------------ */
#define SDFO_FILE_ANY 0    /* SdfOracle::loadFromFile (SdfOracle.cpp:165-172):
                              sparse when isSparseSdf, else dense */
#define SDFO_FILE_DENSE 1  /* loadSdf */
#define SDFO_FILE_SPARSE 2 /* loadSparseSdf */

/* isValidSdf / isSparseSdf (SdfIO.cpp:527-550): reads the 128-byte header
 * only (no device work); a missing or short file gives 0 / 0. */
int sdfo_file_probe(const char* path, int32_t* is_valid, int32_t* is_sparse);

/* loadSdf / loadSparseSdf straight into a device grid: the header is checked
 * with the reference's messages (SDFO_ERR_IO, sdfo_last_error), the payload
 * is read by up to 4 threads through pinned staging and decoded on the device
 * (dense: FP64 arrays kept for exact export plus the FP32 query payload;
 * sparse: FP32 bricks, Hessians if stored, block table; contact-aware
 * candidates when the file has them).  The 64 MiB of pinned staging is
 * allocated on first use and held until the process exits; calls serialise.
 * sdfo_grid_build_stats of the new grid reports the load's phases: setup_ms
 * (allocation), fill_ms (file read and transfer), hessian_ms (decoding on the
 * device), total_ms.  Synchronous. */
int sdfo_grid_load_file(const char* path, int32_t expect, void* stream, sdfo_grid** out);

/* saveSdf / saveSparseSdf of a device grid: byte-identical to the reference
 * writing the same data (dense files always carry Hessians, zero when the
 * grid has none; FP16 grids are written decoded to FP32).  SDFO_ERR_IO when
 * the file cannot be opened or written.  Synchronous. */
int sdfo_grid_save_file(const sdfo_grid* g, const char* path, void* stream);

/* ---- queries (SdfOracle::queryFast / queryBatch) ------------------------- */
/* SdfOracle::queryFast + queryBatch (SdfOracle.cpp:226-444) for n points.
 * d_points: (n,3) float32 or float64 (points_f64).  Outputs (device, any may
 * be NULL except d_gap):
 *   d_gap[n]          interpolated signed distance ("gap")
 *   d_grad[n*3]       raw gradient of the interpolant (FirstOrder: n0;
 *                     SecondOrder: n0 + H0 dx, as the reference's normal)
 *   d_unit[n*3]       the reference's gapNormal: grad/|grad|, UnitX when
 *                     |grad| <= 1e-15 (SecondOrder: falls back to n0)
 *   d_witness[n*3]    p - gap * gapNormal
 *   d_valid[n]        1 if the query is inside the stored domain
 *   d_hess[n*9]       d grad / d p of the interpolant (row-major), the
 *                     forward-mode Jacobian of (gap, grad) w.r.t. p
 * Invalid queries write gap 0, grad 0, unit (1,0,0), witness 0, hess 0.
 * ContactAware on a grid with surface-feature candidates (built by
 * sdfo_grid_build_contact_aware, loaded, or attached) answers with the
 * candidate of smallest |gap| at the nearest voxel (SdfOracle.cpp:296-423);
 * on grids without candidates it behaves as Tricubic, as the reference does
 * (SdfOracle.cpp:209-212). */
int sdfo_query(const sdfo_grid* g, int32_t mode, const void* d_points, int32_t points_f64,
               int64_t n, float* d_gap, float* d_grad, float* d_unit, float* d_witness,
               uint8_t* d_valid, float* d_hess, void* stream);

/* Same with host buffers (pageable or pinned): copies in, queries, copies
 * out; synchronous.  With pinned buffers and more than
 * sdfo_tuning.host_chunk_queries points the batch runs as a pipeline over
 * growing chunks: copies in on `stream`, queries and copies out on two
 * streams of the handle, so that both directions of the bus are busy at
 * once.  Calls on one
 * handle serialise.  Returns SDFO_ERR_DEVICE_STATUS when the pipelined query
 * kernel reports a wait that ran out (see sdfo_device_status). */
int sdfo_query_host(const sdfo_grid* g, int32_t mode, const void* h_points, int32_t points_f64,
                    int64_t n, float* h_gap, float* h_grad, float* h_unit, float* h_witness,
                    uint8_t* h_valid, void* stream);

/* sdfo_query_host without any device allocation.  No counterpart in the
 * reference.  For callers that cannot let a library allocate device memory
 * (applications that give all GPU memory to their own pool at start-up, or
 * that forbid cudaMalloc and the synchronisation it implies inside their
 * step loop): the host points and results are staged through one fixed
 * device array of SDFO_STATIC_STAGING_BYTES that is part of the library image
 * -- every GPU that loads libsdfo_cuda holds it until the process exits.
 * Outputs: h_gap (required), h_grad and h_valid (may be NULL); points and
 * outputs together must fit the array (about 1.1M float32 queries with all
 * outputs), larger batches return SDFO_ERR_INVALID_ARGUMENT.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress) and
 * should come before any stream capture.  Every call shares the array and
 * leaves its contents behind: calls that overlap on the GPU (from several
 * host threads or streams at once) race on it, so callers must serialise
 * them.  Synchronous; the grid's device must be current.  Returns
 * SDFO_ERR_DEVICE_STATUS, and no results, when the pipelined query kernel
 * reports a wait that ran out (see sdfo_device_status). */
#define SDFO_STATIC_STAGING_BYTES (32u << 20)
int sdfo_query_host_static(const sdfo_grid* g, int32_t mode, const void* h_points,
                           int32_t points_f64, int64_t n, float* h_gap, float* h_grad,
                           uint8_t* h_valid, void* stream);

/* Backward of sdfo_query (no reference counterpart): given upstream
 * d_dgap[n] and d_dgrad[n*3] (either may be NULL = zero), writes
 *   d_dpoints[n*3] = dgap * grad + H * dgrad        (may be NULL)
 * and accumulates into d_dgrid (float4 per stored voxel: d phi, d n) the
 * gradient w.r.t. the stored payload (may be NULL; for FP16 storage, w.r.t.
 * the decoded values).  Trilinear and Tricubic; float32 points. */
int sdfo_query_backward(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                        const float* d_dgap, const float* d_dgrad, float* d_dpoints,
                        float* d_dgrid, void* stream);

/* Forward of the differentiable query (no reference counterpart):
 * sdfo_query on float32 points that also writes, per point, the symmetric
 * Hessian of the interpolant d_hess6[n*6] = {xx, xy, xz, yy, yz, zz} (zero
 * where invalid) -- the local linearisation that reverse mode needs, so
 * that sdfo_query_backward_saved reads 24 bytes per point instead of the
 * grid stencil.  d_gap, d_grad, d_valid and d_hess6 are required.
 * Trilinear and Tricubic. */
int sdfo_query_linearize(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                         float* d_gap, float* d_grad, uint8_t* d_valid, float* d_hess6,
                         void* stream);

/* Backward from the linearisation of sdfo_query_linearize (same grid, mode
 * and points):
 *   d_dpoints[n*3] = dgap * grad + H * dgrad     (needs d_grad, d_hess6)
 *   d_dgrid       += dL/d(stored {phi, n})       (needs d_points, d_valid)
 * Either output may be NULL; d_dgap / d_dgrad may be NULL (= zero).  The
 * grid gradient uses only the corner weights at each point, so it is
 * defined for FP32 and FP16 storage alike (w.r.t. the decoded values). */
int sdfo_query_backward_saved(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                              const float* d_grad, const float* d_hess6, const uint8_t* d_valid,
                              const float* d_dgap, const float* d_dgrad, float* d_dpoints,
                              float* d_dgrid, void* stream);

/* SdfFastQueryResult's candidate list (SdfCommon.h:29-37) for every point:
 * d_ncand (n) int32, d_kgap (n*8), d_knormal (n*8*3), d_kwitness (n*8*3)
 * float32, d_kbranch (n*8) int32 (slots past ncand: gap 0, normal (1,0,0),
 * witness 0, branch -1).  ContactAware on a grid with candidates: each of
 * the voxel's candidates extrapolated linearly, gap = phi + n.(p - centre)
 * (SdfOracle.cpp:296-423); otherwise one candidate, the query's own result
 * with branch 0 (fastFromQueryResult, SdfOracle.cpp:86-120).  Invalid
 * points: ncand 0.  The main results go to d_gap / d_normal (gapNormal) /
 * d_witness / d_valid; every output is required; float32 points. */
int sdfo_query_candidates(const sdfo_grid* g, int32_t mode, const float* d_points, int64_t n,
                          float* d_gap, float* d_normal, float* d_witness, uint8_t* d_valid,
                          int32_t* d_ncand, float* d_kgap, float* d_knormal, float* d_kwitness,
                          int32_t* d_kbranch, void* stream);
/* sdfo_query_candidates with host buffers (points float32 or float64 per
 * points_f64); synchronous.  The C++ SdfOracle::queryFast / query /
 * queryBatch fill their candidate lists from it. */
int sdfo_query_candidates_host(const sdfo_grid* g, int32_t mode, const void* h_points,
                               int32_t points_f64, int64_t n, float* h_gap, float* h_normal,
                               float* h_witness, uint8_t* h_valid, int32_t* h_ncand,
                               float* h_kgap, float* h_knormal, float* h_kwitness,
                               int32_t* h_kbranch, void* stream);

/* ---- batched queries over many grids (no reference counterpart) --------- */
/* Rigid placement of a grid in the world: x_world = R x_grid + t (R
 * row-major).  A query point p is looked up at R^T (p - t) (FP64) and its
 * gradient returned in the world frame, R grad. */
typedef struct
{
    double R[9];
    double t[3];
} sdfo_pose;

typedef struct sdfo_query_batch sdfo_query_batch;

/* A fixed layout of queries over n grids: grid g answers h_counts[g]
 * consecutive points (grids in order).  The grids must outlive the batch
 * and stay on one device.  Uploads the grid descriptors once, so that
 * sdfo_query_batch_run allocates nothing and can be captured in a CUDA
 * graph. */
int sdfo_query_batch_create(const sdfo_grid* const* grids, int32_t n, const int64_t* h_counts,
                            sdfo_query_batch** out);
/* One launch over all grids' queries: d_points (total, 3) float32 world
 * points; d_poses (n) device array or NULL (identity); outputs d_gap
 * (total), d_grad (total, 3, world frame, may be NULL), d_valid (total, may
 * be NULL).  Trilinear or Tricubic; dense and sparse (FP32 / FP16) grids
 * may be mixed.  Asynchronous on `stream`. */
int sdfo_query_batch_run(const sdfo_query_batch* b, int32_t mode, const float* d_points,
                         const sdfo_pose* d_poses, float* d_gap, float* d_grad, uint8_t* d_valid,
                         void* stream);
/* Launch shape of sdfo_query_batch_run: threads per CTA, 128 (default), 256
 * or 512 -- a knob the autotuner sets. */
int sdfo_query_batch_set_threads(sdfo_query_batch* b, int32_t threads);
/* Tile order of sdfo_query_batch_run: each persistent CTA takes `tiles`
 * consecutive tiles (a power of two, 1..64; default 4) before it strides by
 * the launch's CTA count, so the resident CTAs work on a window of
 * consecutive tiles (a few grids, whose brick pools then stay in L2). */
int sdfo_query_batch_set_run(sdfo_query_batch* b, int32_t tiles);
int sdfo_query_batch_total(const sdfo_query_batch* b, int64_t* total);
int sdfo_query_batch_destroy(sdfo_query_batch* b);

/* ---- contact (SDFContactEngine.evaluate) --------------------------------- */
/* Batched SDFContactEngine.evaluate (prototype/src/dynamics/contacts_sdf.py:
 * 225-385) for P poses of body A (the quadrature body) against the grid of
 * body B: Y = R_B^T R_A X + R_B^T (r_A - r_B); penalty p = k max(-g,0)^n
 * along R_B grad g; damping c (-v_n) R_B grad g when g < 0; regularised
 * Coulomb friction -mu p |grad g| u_t / sqrt(|u_t|^2 + reg^2).
 *   d_quad_x (Q,3) float32 body-A-local points, d_quad_w (Q) float32 weights
 *   d_pose_a (P) body A states, d_body_b (1) body B state (device)
 *   d_ft (P,6) float64: F_A, tau_A (tau about r_A)
 *   d_jac (P,36) float64 or NULL: row-major d(F_A,tau_A)/d(dx,dtheta) for
 *   r_A += dx, R_A = exp([dtheta]x) R_A (forward-mode, in-kernel).
 * Mode: Trilinear or Tricubic. */
int sdfo_contact_eval(const sdfo_grid* g, int32_t mode, const float* d_quad_x,
                      const float* d_quad_w, int64_t nq, const sdfo_body_state* d_pose_a,
                      int64_t np, const sdfo_body_state* d_body_b,
                      const sdfo_contact_params* h_params, double* d_ft, double* d_jac,
                      void* stream);

/* ---- contact pairs with the engine's culling ---------------------------- */
typedef struct sdfo_contact_pair sdfo_contact_pair;

/* SDFContactEngine.register_pair (contacts_sdf.py:52-62): quadrature points
 * (nq,3) FP64 in body A's frame and their weights (normalised to sum 1 when
 * normalize_weights != 0), bound to grid g (which must outlive the pair),
 * with the AABB_BVH point hierarchy (geometry/bvh.py:16-60, leaf_size 16 in
 * the reference).  narrow_margin >= 0 enables the engine's culling with that
 * narrow margin (0.01 in the reference): the BVH cull with box margin
 * max(narrow_margin, 0.05) and evaluate's |Y_z| < narrow_margin filter;
 * narrow_margin < 0 evaluates every point.  At most 32768 BVH leaves when
 * culling is enabled (SDFO_ERR_UNSUPPORTED beyond).  g == NULL builds the
 * hierarchy only, on the host (for sdfo_contact_pair_export_bvh). */
int sdfo_contact_pair_create(const sdfo_grid* g, const double* h_quad_x, const double* h_quad_w,
                             int64_t nq, int32_t normalize_weights, double narrow_margin,
                             int32_t leaf_size, sdfo_contact_pair** out);

/* The pair's point hierarchy: leaf count, the original point indices in
 * stored order (nq), leaf offsets into that order (nleaves + 1) and leaf
 * boxes (nleaves x 6: min xyz, max xyz).  Leaves are in the order the
 * reference's query visits them.  Any output may be NULL. */
int sdfo_contact_pair_export_bvh(const sdfo_contact_pair* p, int32_t* h_nleaves,
                                 int32_t* h_point_order, int32_t* h_leaf_start,
                                 double* h_leaf_box);

/* evaluate (contacts_sdf.py:225-385) and/or measure_pair
 * (contacts_sdf.py:171-214) for np poses of body A against body B: d_ft
 * (np x 6: F_A, tau_A), d_jac (np x 36, as sdfo_contact_eval; needs d_ft) and
 * d_measure (np) -- any of them may be NULL, not all. */
int sdfo_contact_pair_eval(const sdfo_contact_pair* p, int32_t mode,
                           const sdfo_body_state* d_pose_a, int64_t np,
                           const sdfo_body_state* d_body_b, const sdfo_contact_params* h_params,
                           double* d_ft, double* d_jac, sdfo_contact_measure* d_measure,
                           void* stream);

int sdfo_contact_pair_destroy(sdfo_contact_pair* p);

/* ---- Backward-Euler contact steps ---------------------------------------- */
/* Newton tangent of the BE solve (sdfo_be_params.tangent).
 * REFERENCE: the reference's method -- contact forces inside a step reuse
 *   the linearisation cache g + grad . dt of its first evaluation
 *   (contacts_sdf.py:306-326) and Newton uses the heuristic diagonal contact
 *   stiffness (_contact_tangent / _tangent, implicit_be.py:606-687).
 * EXACT (no reference counterpart): every residual evaluates contact exactly
 *   and Newton uses the analytic dR/dV -- M/h, the rotational inertia and
 *   gyroscopic terms differentiated through R(w), and the contact block
 *   Jv + Jp diag(h I, h J_l(h w)) from the force law differentiated per
 *   quadrature point (Jp: w.r.t. the pose, R <- exp([dtheta]x) R, at fixed
 *   velocities; Jv: w.r.t. (v, w) at a fixed pose; J_l the SO(3) left
 *   Jacobian).  It converges to the exact BE solution of each step. */
#define SDFO_BE_TANGENT_REFERENCE 0
#define SDFO_BE_TANGENT_EXACT 1

/* BackwardEulerIntegrator parameters (implicit_be.py:60-107 defaults via
 * sdfo_be_params_default). */
typedef struct
{
    int32_t max_iter;            /* 20 */
    int32_t line_search;         /* 1 */
    int32_t max_toi_bisect_iter; /* 60 */
    int32_t stable_steps;        /* contact_stable_steps, 5 */
    int32_t release_steps;       /* contact_release_steps, 3 */
    int32_t tangent;             /* SDFO_BE_TANGENT_*, default REFERENCE */
    double tol;                  /* 1e-8 */
    double pen_max;              /* contact_penetration_tol, 1e-6 */
    double dt_min;               /* contact_dt_min, 1e-8 */
    double dt_impact;            /* contact_dt_impact, 1e-7 */
    double dt_contact;           /* contact_dt_active, 1e-5 */
    double dt_max_contact;       /* contact_dt_max, 1e-4 */
    double dt_normal;            /* contact_dt_normal, 1e-3 */
    double dt_growth;            /* contact_dt_growth, 1.5 */
} sdfo_be_params;

/* RigidBody mass properties (ir/body.py): mass, body-frame inertia
 * (row-major 3x3), and the model's gravity. */
typedef struct
{
    double mass;
    double inertia[9];
    double gravity[3];
} sdfo_rigid_body;

/* One scene: the state of body A and its contact region
 * (ContactRegionState, implicit_be.py:22-39; phase numbered as ContactPhase:
 * 0 INACTIVE, 2 IMPACTING, 3 ACTIVE, 4 STABLE, 5 LEAVING). */
typedef struct
{
    sdfo_body_state body;
    double t;
    double dt_current;
    double last_gap;
    double last_penetration;
    double last_normal_velocity;
    double last_toi;
    int32_t phase;
    int32_t stable_count;
    int32_t release_count;
    int32_t min_dt_hits;
} sdfo_be_scene;

typedef struct sdfo_be_stepper sdfo_be_stepper;

void sdfo_be_params_default(sdfo_be_params* p);
/* A scene at rest in the state machine: INACTIVE, dt_current = dt_normal,
 * last_gap and last_toi +inf (ContactRegionState defaults). */
void sdfo_be_scene_init(sdfo_be_scene* s, const sdfo_body_state* body, double t,
                        const sdfo_be_params* p);

/* BackwardEulerIntegrator.step (implicit_be.py:131-181) for batches of
 * scenes: body A (free, mass properties body_a) carries the pair's
 * quadrature set; body B (fixed, state body_b) carries the pair's grid,
 * which must be dense with FP64 values.  The engine's culling follows the
 * pair's narrow margin, its linearisation cache is used as the reference
 * uses it.  Holds scratch for max_scenes scenes (40 B per scene and
 * quadrature point). */
int sdfo_be_stepper_create(const sdfo_contact_pair* pair, const sdfo_contact_params* contact,
                           const sdfo_rigid_body* body_a, const sdfo_body_state* body_b,
                           const sdfo_be_params* params, int64_t max_scenes,
                           sdfo_be_stepper** out);

/* One step of every scene: d_scenes (n, device) advanced in place, d_dt (n)
 * the requested step (<= 0: the scene is left as it is), d_h (n, may be NULL)
 * the step taken (the time of impact when contact begins).  Asynchronous. */
int sdfo_be_stepper_step(sdfo_be_stepper* st, sdfo_be_scene* d_scenes, int64_t n,
                         const double* d_dt, double* d_h, void* stream);

/* Threads per scene: 256 (default; one CTA per scene, three scenes per SM),
 * 128 (four scenes per SM) or 32 (one warp per scene, 24 per SM).  On
 * 2048 drops of a 7,680-point ring, 128 and 256 run within 5 % of each other
 * and 32 takes twice as long (its point passes are 8x longer); 32 suits
 * small quadrature sets. */
int sdfo_be_stepper_set_threads(sdfo_be_stepper* st, int32_t threads);

/* BackwardEulerIntegrator.integrate (implicit_be.py:113-129), `launches`
 * steps of it for every scene: a scene with t < t_end - 1e-15 (d_t_end (n),
 * device) takes one step of at most min(dt, t_end - t), with the loop's
 * zero-progress fail-safe (a plain BE step of min(dt_min, t_end - t) when a
 * step makes no progress); the others are left as they are.  The launches
 * run as one CUDA graph, captured on the first call with a set of arguments
 * and replayed while they stay the same.  d_unfinished (device, may be NULL)
 * receives the number of scenes still short of t_end after the last launch.
 * Asynchronous. */
int sdfo_be_stepper_advance(sdfo_be_stepper* st, sdfo_be_scene* d_scenes, int64_t n,
                            const double* d_t_end, double dt, int32_t launches,
                            int32_t* d_unfinished, void* stream);

/* The whole integrate loop: sdfo_be_stepper_advance of launches_per_check
 * launches, then a 4-byte read of the unfinished count, until every scene
 * has reached t_end or max_launches launches are made.  Synchronises
 * `stream`.  *launches_out: launches made; *unfinished_out: scenes still
 * short of t_end (0 unless max_launches ran out).  Both may be NULL. */
int sdfo_be_stepper_integrate(sdfo_be_stepper* st, sdfo_be_scene* d_scenes, int64_t n,
                              const double* d_t_end, double dt, int32_t launches_per_check,
                              int64_t max_launches, int64_t* launches_out,
                              int32_t* unfinished_out, void* stream);

/* Work counters summed over every launch since creation or the last reset
 * (no reference counterpart): out[0] Newton iterations, out[1] residual
 * evaluations, out[2] BE solves (_step_be calls, trial steps included).
 * Synchronises the device; reset != 0 zeroes them after the read. */
int sdfo_be_stepper_stats(sdfo_be_stepper* st, uint64_t* out, int32_t reset);

int sdfo_be_stepper_destroy(sdfo_be_stepper* st);

#ifdef __cplusplus
}
#endif
#endif /* SDFO_H */
