// Internal declarations shared by the libsdfo_cuda translation units.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "sdfo.h"

namespace sdfo {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
struct Error
{
    int code;
    std::string msg;
    Error(int c, std::string m) : code(c), msg(std::move(m)) {}
};

void set_last_error(const std::string& msg);

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);

#define SDFO_CUDA(call)                                                                  \
    do                                                                                   \
    {                                                                                    \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) ::sdfo::throw_cuda(e_, #call, __FILE__, __LINE__);        \
    } while (0)

#define SDFO_CHECK_LAUNCH() SDFO_CUDA(cudaGetLastError())

#define SDFO_REQUIRE(cond, code, msg)                                                    \
    do                                                                                   \
    {                                                                                    \
        if (!(cond)) throw ::sdfo::Error((code), (msg));                                 \
    } while (0)

// Runs f() and converts exceptions into a status code + last-error message.
template <class F>
int guarded(F&& f)
{
    try
    {
        f();
        return SDFO_OK;
    }
    catch (const Error& e)
    {
        set_last_error(e.msg);
        return e.code;
    }
    catch (const std::bad_alloc&)
    {
        set_last_error("host out of memory");
        return SDFO_ERR_OUT_OF_MEMORY;
    }
    catch (const std::exception& e)
    {
        set_last_error(e.what());
        return SDFO_ERR_INVALID_ARGUMENT;
    }
}

// Multiprocessor count of device `dev`, looked up once per device
// (thread-safe; grid.cu).
int device_sm_count(int dev);
// ... of the current device.
int current_sm_count();

// Device allocation owned by a grid handle.
void* device_alloc(size_t bytes);
void device_free(void* p);

// Limit (bytes per device; < 0 leaves it, 0 releases all and disables) and
// current size of the cache of freed device blocks (grid.cu).
void device_cache_control(int64_t limit, int64_t* held);

template <class T>
T* dalloc(size_t count)
{
    return static_cast<T*>(device_alloc(count * sizeof(T)));
}

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

// Scoped device buffer for temporaries inside one call.
template <class T>
struct DeviceBuffer
{
    T* p = nullptr;
    size_t n = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t count) { reset(count); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { device_free(p); }
    void reset(size_t count)
    {
        device_free(p);
        p = count ? dalloc<T>(count) : nullptr;
        n = count;
    }
    T* get() const { return p; }
};

// ---------------------------------------------------------------------------
// grid storage
// ---------------------------------------------------------------------------
// Device payload of a grid.  Dense: one float4 {phi, n} per voxel, x-fastest,
// plus optional FP32 Hessians and the FP64 build results for exact export.
// Sparse: bricks of block_dim^3 voxels in stored order (local index
// lx + bd*(ly + bd*lz)), a dense int32 table over block coordinates, and the
// block coordinates.  FP16 sparse storage keeps {phi_q, nx, ny, nz} as four
// halves per voxel and a float2 {scale, offset} per brick.
struct GridStorage
{
    float4* phin = nullptr;
    float* hess6 = nullptr;
    double* phi64 = nullptr;
    double* n64 = nullptr;
    double* w64 = nullptr;
    double* h64 = nullptr;
    int32_t* table = nullptr;
    int32_t* ijk = nullptr;
    ushort4* phin16 = nullptr;
    float2* brick_affine = nullptr;
    float4* xpair = nullptr; // 2 float4 per voxel
    float4* cell8 = nullptr; // 2 float4 per voxel
    // contact-aware candidates, `stride` slots per stored voxel: count (u8),
    // phi and normal (FP64 for dense grids, FP32 for sparse ones, as the
    // reference stores them), branch id
    uint8_t* ca_count = nullptr;
    double* ca_phi64 = nullptr;
    double* ca_n64 = nullptr;
    float* ca_phi32 = nullptr;
    float* ca_n32 = nullptr;
    int32_t* ca_branch = nullptr;
};

// Streams, events and the pinned status word of the chunked host-buffer
// query path (capi.cu), created on a handle's first host query.
struct HostPipe;
void destroy_host_pipe(HostPipe* p);

} // namespace sdfo

struct sdfo_grid
{
    sdfo_grid_info info{};
    sdfo::GridStorage d{};
    sdfo_build_stats stats{};
    int device = 0;
    int64_t stored_voxels = 0;
    int32_t nb[3] = {0, 0, 0};
    int ca_stride = 0;      // contact-aware candidate slots per voxel (0 = none)
    bool borrowed = false; // a view: storage belongs to another handle / caller
    // Storage shared by the grids of one batched build (released with the
    // last of them); empty otherwise.
    std::shared_ptr<void> arena;
    // Device staging for the host-buffer query path, grown on demand and
    // reused across calls; calls on one handle serialise on the mutex.
    mutable std::mutex ws_mutex;
    mutable void* ws = nullptr;
    mutable size_t ws_bytes = 0;
    mutable sdfo::HostPipe* host_pipe = nullptr;
    ~sdfo_grid();
};

// A contact pair (contact_pair.cu): the quadrature set of body A bound to
// body B's grid, with its point hierarchy.  Points are stored leaf by leaf
// (px, pw, porig, pleaf) in FP32 for the contact kernels and in FP64 (px64,
// pw64) for the BE step, which also keeps them in their original order
// (ox64, ow64).
struct sdfo_contact_pair
{
    const sdfo_grid* grid = nullptr;
    int64_t nq = 0;
    double narrow_margin = -1.0;
    int nleaves = 0;
    double root[6] = {0, 0, 0, 0, 0, 0};
    std::vector<int32_t> h_order, h_leaf_start;
    std::vector<double> h_leaf_box;
    float* px = nullptr;
    float* pw = nullptr;
    double* px64 = nullptr;
    double* pw64 = nullptr;
    double* ox64 = nullptr;
    double* ow64 = nullptr;
    int32_t* porig = nullptr;
    int32_t* pleaf = nullptr;
    int32_t* leaf_start = nullptr;
    double* leaf_box = nullptr;
    ~sdfo_contact_pair();
};

namespace sdfo {

// Largest m in [0, n) with offs[m] <= x (offs non-decreasing, offs[0] = 0):
// the segment of a concatenation that holds element x, skipping empty
// segments.
__device__ __forceinline__ int find_segment(const int64_t* __restrict__ offs, int n, int64_t x)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(offs + mid) <= x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Kernel-side view of a grid (passed by value).
struct GridView
{
    double bmin[3];
    double voxel[3];
    double ivoxel[3]; // 1 / voxel (FP64)
    float ih[3];      // 1 / voxel (FP32)
    int nx, ny, nz;
    int layout;  // SDFO_LAYOUT_*
    int storage; // SDFO_STORAGE_*
    int phin_a32; // the query payload (phin, or phin16 for FP16 storage) starts on a
                  // 32-byte boundary: 256-bit loads of sparse brick rows
    int has_hessian;
    const float4* phin;
    const float* hess6;
    const int32_t* table;
    int nbx, nby, nbz;
    int bd;
    const ushort4* phin16;
    const float2* brick_affine;
    // Dense stencil layouts (32-byte records, one 256-bit load each), or NULL:
    //   xpair[v] = {phin[v], phin[v + 1]}             Tricubic: 4 loads / query
    //   cell8[v] = phi of the 8 corners of cell v       Trilinear: 1 load / query
    const float4* xpair;
    const float4* cell8;
    // contact-aware candidates (ca_stride == 0: none)
    int ca_stride;
    const uint8_t* ca_count;
    const double* ca_phi64;
    const double* ca_n64;
    const float* ca_phi32;
    const float* ca_n32;
    const int32_t* ca_branch;
};

GridView make_view(const sdfo_grid* g);
// Which sparse 8^3-brick FP32 grids created from now on get x-pair records
// (2x the payload's memory): 0 those with pools up to 48 MB, 1 all, 2 none
// (grid.cu).
int sparse_pair_records();
void set_sparse_pair_records(int mode);
// FP32-point queries by the persistent walk kernel (query.cu)
bool query_walk();
void set_query_walk(bool on);
// Fills the stencil layouts from phin (grid.cu): dense xpair and cell8;
// sparse 8^3 FP32 bricks: xpair as sparse_pair_records() selects.
void build_stencil_layouts(sdfo_grid* g, cudaStream_t s);

// Query launch (query.cu).
struct QueryOutputs
{
    float* gap;
    float* grad;
    float* unit;
    float* witness;
    uint8_t* valid;
    float* hess;            // 9 per query (full 3x3), or NULL
    float* hess6 = nullptr; // 6 per query (xx, xy, xz, yy, yz, zz), or NULL
    // outputs live in host memory mapped into the device: plain stores only
    // (no bulk-copy stores)
    bool host_mapped = false;
};
void launch_query(const GridView& v, int mode, const void* pts, bool f64, int64_t n,
                  const QueryOutputs& o, cudaStream_t s);
// Candidate lists of SdfFastQueryResult (NULL kgap: not written).
struct CandidateOutputs
{
    int32_t* ncand;
    float* kgap;
    float* knormal;
    float* kwitness;
    int32_t* kbranch;
};
// Status bits of the pipelined query kernel (query.cu), read and optionally
// cleared by sdfo_device_status.
unsigned query_pipe_status(bool clear);
// Device address of that status word on the current device (looked up once
// per device), for stream-ordered reads by the synchronous host paths.
unsigned* query_pipe_status_address();
// Bit of the status word that k_query_pipe sets when a bounded wait runs out.
constexpr unsigned kPipeStatusWaitAbort = 2u;
// Test-only settings of the bounded waits (query.cu, stream_bwd.cu): the
// main-loop wait limit in try-wait iterations (0 = the built-in limit) and
// whether every CTA withholds the bulk load of its first tile, so that the
// wait for it can only run out.  Process-wide; 0, 0 restores normal
// operation.
void set_query_pipe_wait_test(unsigned limit, int withhold_first_tile);
void set_backward_bulk_wait_test(unsigned limit, int withhold_first_tile);
// dL/dp of the saved backward for all n queries as a bulk-copy pipeline
// (stream_bwd.cu); false (nothing launched) when n < 256 or the pointers are
// not 16-byte aligned.
bool launch_backward_saved_bulk(int64_t n, const float* grad, const float* hess6, const float* dgap,
                                const float* dgrad, float* dpts, cudaStream_t s);
// ContactAware on a grid with candidates (ca_query.cu).
void launch_query_ca(const GridView& v, const void* pts, bool f64, int64_t n, const QueryOutputs& o,
                     const CandidateOutputs& co, cudaStream_t s);
void launch_single_candidate(int64_t n, const float* gap, const float* unit, const float* wit,
                             const uint8_t* valid, const CandidateOutputs& co, cudaStream_t s);
void launch_query_backward(const GridView& v, int mode, const float* pts, int64_t n,
                           const float* dgap, const float* dgrad, float* dpts, float* dgrid,
                           cudaStream_t s);

// Reverse mode from a saved linearisation (query.cu).
struct SavedBackward
{
    const float* pts;
    int64_t n;
    const float* grad;
    const float* hess6;
    const uint8_t* valid;
    const float* dgap;
    const float* dgrad;
    float* dpts;
    float* dgrid;
};
void launch_backward_saved(const GridView& v, int mode, const SavedBackward& b, cudaStream_t s);

// Builders (build.cu).
sdfo_grid* build_dense(const double* verts, int64_t nv, const int32_t* tris, int64_t nt,
                       const sdfo_build_params& p, cudaStream_t s);
sdfo_grid* build_sparse(const double* verts, int64_t nv, const int32_t* tris, int64_t nt,
                        const sdfo_sparse_build_params& p, cudaStream_t s);
sdfo_grid_info setup_grid(const double* verts, int64_t nv, const sdfo_build_params& p);
// The dense fill's traversals counted over the grid of p (build.cu).
void count_dense_traversal(const double* verts, int64_t nv, const int32_t* tris, int64_t nt,
                           const sdfo_build_params& p, cudaStream_t s, sdfo_traversal_stats* out);
// Batched sparse build (batch.cu): one grid per mesh, storage in one arena.
std::vector<sdfo_grid*> build_sparse_batched(const sdfo_mesh_desc* meshes, int n, cudaStream_t s);
void set_fill_ctas_per_sm(int k);
int fill_ctas_per_sm();
// Contact-aware build (ca_build.cu).
sdfo_grid* build_contact_aware(const double* verts, int64_t nv, const int32_t* tris, int64_t nt,
                               const double* cnormals, const sdfo_contact_aware_params& p,
                               cudaStream_t s);
int bvh_mode();
void set_bvh_mode(int m);
// Inside/outside sign rule of subsequent builds (build.cu).
int sign_mode();
void set_sign_mode(int m);
// Voxel tile of the dense fill CTAs, as log2 extents in x and y (z takes the
// rest of 256 threads); 0 selects the default 3 (8 x 8 x 4) (build.cu).
void set_fill_tile(int lx, int ly);
void get_fill_tile(int* lx, int* ly);
// LBVH traversals by parent links instead of a per-thread stack (build.cu).
int lbvh_stackless();
void set_lbvh_stackless(int on);
// The FP32 triangle-box cull ahead of the FP64 closest-point test of the
// reference-order tree (build.cu; on by default).
int triangle_cull();
void set_triangle_cull(int on);

// Contact (contact.cu).
// The culling of SDFContactEngine.evaluate / measure_pair: a point BVH over
// the quadrature points (leaves in the order the reference's query visits
// them, points stored leaf by leaf), the query box margin and the |Y_z|
// narrow filter.  enabled == 0: every point, in its stored order.
constexpr int kMaxCullLeaves = 32768;
struct ContactCull
{
    int enabled;
    int nleaves;
    const double* leaf_box;   // (nleaves, 6): min x y z, max x y z
    const int32_t* leaf_start; // (nleaves + 1) offsets into the point order
    const int32_t* pleaf;      // leaf of each stored point
    const int32_t* porig;      // original index of each stored point
    double root[6];            // box of all points
    double bmin[3], bmax[3];   // the grid's box (sdf.bmin / sdf.bmax)
    double box_margin;         // max(narrow_margin, 0.05)
    double narrow_margin;      // evaluate keeps |Y_z| < narrow_margin
};
void launch_contact(const GridView& v, int mode, const float* qx, const float* qw, int64_t nq,
                    const sdfo_body_state* pose_a, int64_t np, const sdfo_body_state* body_b,
                    const sdfo_contact_params& prm, double* ft, double* jac, cudaStream_t s,
                    const ContactCull* cull = nullptr, sdfo_contact_measure* meas = nullptr);

// FP16 re-encoding (grid.cu).
void encode_fp16(const sdfo_grid* src, sdfo_grid* dst, cudaStream_t s);

} // namespace sdfo
