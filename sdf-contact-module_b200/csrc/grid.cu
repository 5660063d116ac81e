// Grid handles: creation from host SdfData / SparseSdfData arrays, export,
// device views and the FP16 re-encoding of sparse payloads.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "sdfo_internal.cuh"

namespace sdfo {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }

void throw_cuda(cudaError_t e, const char* what, const char* file, int line)
{
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e,
                  cudaGetErrorString(e), what, file, line);
    if (e == cudaErrorMemoryAllocation) throw Error(SDFO_ERR_OUT_OF_MEMORY, buf);
    throw Error(SDFO_ERR_CUDA, buf);
}

// ---------------------------------------------------------------------------
// Multiprocessor counts, one slot per device ordinal, filled on first use.
// Two threads filling the same slot store the same value; the slots are
// atomics so that the unsynchronised read is well defined.
// ---------------------------------------------------------------------------
namespace {
constexpr int kMaxSmDevices = 64;
std::atomic<int> g_sm_count[kMaxSmDevices];
} // namespace

int device_sm_count(int dev)
{
    SDFO_REQUIRE(dev >= 0 && dev < kMaxSmDevices, SDFO_ERR_UNSUPPORTED, "device ordinal too large");
    int v = g_sm_count[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    SDFO_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    g_sm_count[dev].store(v, std::memory_order_relaxed);
    return v;
}

int current_sm_count()
{
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    return device_sm_count(dev);
}

// ---------------------------------------------------------------------------
// Device memory: cudaMalloc and cudaFree each cost about 0.3 ms whatever the
// size, and a build makes a dozen of them.  Freed blocks are therefore kept
// per device, by size class, and handed out again for a request of the same
// class.  A free first synchronises the device, as cudaFree does, so no block
// is handed out while work queued before its free can still touch it.
// ---------------------------------------------------------------------------
namespace {

struct Live
{
    size_t bytes;
    int device;
};

struct Cache
{
    std::mutex mu;
    std::unordered_map<void*, Live> live;              // handed out
    std::vector<std::vector<std::pair<void*, size_t>>> free_blocks; // per device, oldest first
    std::vector<size_t> held;                           // per device
    int64_t limit = int64_t(1) << 30;                   // per device
};

Cache& cache()
{
    static Cache* c = new Cache(); // never destroyed: frees may run during exit
    return *c;
}

// Size class: powers of two up to 2 MiB, then multiples of 2 MiB.
size_t size_class(size_t b)
{
    const size_t mb2 = size_t(2) << 20;
    if (b >= mb2) return (b + mb2 - 1) / mb2 * mb2;
    size_t c = 512;
    while (c < b) c <<= 1;
    return c;
}

void ensure_device(Cache& c, int dev)
{
    if ((int)c.free_blocks.size() <= dev)
    {
        c.free_blocks.resize((size_t)dev + 1);
        c.held.resize((size_t)dev + 1, 0);
    }
}

// cudaFree of every cached block of `dev` (the current device) above `keep`
// bytes, oldest first; the caller holds the lock.
void trim_locked(Cache& c, int dev, size_t keep)
{
    auto& fl = c.free_blocks[(size_t)dev];
    size_t i = 0;
    while (c.held[(size_t)dev] > keep && i < fl.size())
    {
        cudaFree(fl[i].first);
        c.held[(size_t)dev] -= fl[i].second;
        ++i;
    }
    fl.erase(fl.begin(), fl.begin() + (std::ptrdiff_t)i);
}

} // namespace

void* device_alloc(size_t bytes)
{
    if (bytes == 0) return nullptr;
    const size_t cls = size_class(bytes);
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    ensure_device(c, dev);
    auto& fl = c.free_blocks[(size_t)dev];
    for (size_t i = fl.size(); i-- > 0;)
        if (fl[i].second == cls)
        {
            void* p = fl[i].first;
            fl.erase(fl.begin() + (std::ptrdiff_t)i);
            c.held[(size_t)dev] -= cls;
            c.live[p] = Live{cls, dev};
            return p;
        }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, cls);
    if (e == cudaErrorMemoryAllocation && c.held[(size_t)dev] > 0)
    {
        // give the cached blocks back and try once more
        (void)cudaGetLastError();
        trim_locked(c, dev, 0);
        e = cudaMalloc(&p, cls);
    }
    if (e != cudaSuccess)
    {
        (void)cudaGetLastError();
        char buf[160];
        std::snprintf(buf, sizeof(buf), "cudaMalloc of %zu bytes failed: %s", bytes,
                      cudaGetErrorString(e));
        throw Error(e == cudaErrorMemoryAllocation ? SDFO_ERR_OUT_OF_MEMORY : SDFO_ERR_CUDA, buf);
    }
    c.live[p] = Live{cls, dev};
    return p;
}

void device_free(void* p)
{
    if (!p) return;
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    auto it = c.live.find(p);
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    if (it == c.live.end() || it->second.device != dev || c.limit <= 0 ||
        (int64_t)it->second.bytes > c.limit)
    {
        if (it != c.live.end()) c.live.erase(it);
        cudaFree(p);
        return;
    }
    const size_t bytes = it->second.bytes;
    c.live.erase(it);
    // the synchronisation cudaFree would make
    if (cudaDeviceSynchronize() != cudaSuccess)
    {
        (void)cudaGetLastError();
        cudaFree(p);
        return;
    }
    ensure_device(c, dev);
    c.free_blocks[(size_t)dev].emplace_back(p, bytes);
    c.held[(size_t)dev] += bytes;
    trim_locked(c, dev, (size_t)c.limit);
}

void device_cache_control(int64_t limit, int64_t* held)
{
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    Cache& c = cache();
    std::lock_guard<std::mutex> lock(c.mu);
    ensure_device(c, dev);
    if (limit >= 0)
    {
        c.limit = limit;
        trim_locked(c, dev, (size_t)limit);
    }
    if (held) *held = (int64_t)c.held[(size_t)dev];
}

GridView make_view(const sdfo_grid* g)
{
    GridView v{};
    for (int a = 0; a < 3; ++a)
    {
        v.bmin[a] = g->info.bmin[a];
        v.voxel[a] = g->info.voxel[a];
        v.ivoxel[a] = 1.0 / g->info.voxel[a];
        v.ih[a] = (float)(1.0 / g->info.voxel[a]);
    }
    v.nx = g->info.shape[0];
    v.ny = g->info.shape[1];
    v.nz = g->info.shape[2];
    v.layout = g->info.layout;
    v.storage = g->info.storage;
    v.has_hessian = g->info.has_hessian && g->d.hess6 != nullptr;
    v.phin = g->d.phin;
    v.hess6 = g->d.hess6;
    v.table = g->d.table;
    v.nbx = g->nb[0];
    v.nby = g->nb[1];
    v.nbz = g->nb[2];
    v.bd = g->info.block_dim;
    v.phin16 = g->d.phin16;
    v.brick_affine = g->d.brick_affine;
    {
        const void* pool = g->info.storage == SDFO_STORAGE_FP16 ? (const void*)g->d.phin16 : (const void*)g->d.phin;
        v.phin_a32 = pool != nullptr && (reinterpret_cast<uintptr_t>(pool) & 31) == 0;
    }
    v.xpair = g->d.xpair;
    v.cell8 = g->d.cell8;
    v.ca_stride = g->ca_stride;
    v.ca_count = g->d.ca_count;
    v.ca_phi64 = g->d.ca_phi64;
    v.ca_n64 = g->d.ca_n64;
    v.ca_phi32 = g->d.ca_phi32;
    v.ca_n32 = g->d.ca_n32;
    v.ca_branch = g->d.ca_branch;
    return v;
}

namespace {

void check_spec(const sdfo_grid_info* info)
{
    SDFO_REQUIRE(info != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid info is NULL");
    for (int a = 0; a < 3; ++a)
    {
        SDFO_REQUIRE(info->shape[a] > 0, SDFO_ERR_INVALID_ARGUMENT, "grid shape must be positive");
        SDFO_REQUIRE(info->voxel[a] > 0.0 && std::isfinite(info->voxel[a]),
                     SDFO_ERR_INVALID_ARGUMENT, "voxel size must be positive and finite");
        SDFO_REQUIRE(std::isfinite(info->bmin[a]), SDFO_ERR_INVALID_ARGUMENT,
                     "bmin must be finite");
    }
    const int64_t n = (int64_t)info->shape[0] * info->shape[1] * info->shape[2];
    SDFO_REQUIRE(n < (int64_t(1) << 40), SDFO_ERR_INVALID_ARGUMENT, "grid too large");
}

// FP16 brick encoding: per brick, phi is mapped affinely to [-1, 1]
// (offset = mid-range, scale = half-range) and stored as half with the
// normal's three components.
__global__ void k_encode_fp16(const float4* __restrict__ phin, int V, ushort4* __restrict__ out,
                              float2* __restrict__ affine)
{
    const int64_t brick = blockIdx.x;
    const float4* src = phin + brick * V;
    float lo = INFINITY, hi = -INFINITY;
    for (int i = threadIdx.x; i < V; i += blockDim.x)
    {
        const float x = src[i].x;
        lo = fminf(lo, x);
        hi = fmaxf(hi, x);
    }
    __shared__ float slo[32], shi[32];
    for (int o = 16; o > 0; o >>= 1)
    {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
    {
        slo[warp] = lo;
        shi[warp] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 1; w < nw; ++w)
        {
            slo[0] = fminf(slo[0], slo[w]);
            shi[0] = fmaxf(shi[0], shi[w]);
        }
        const float off = 0.5f * (slo[0] + shi[0]);
        float sc = 0.5f * (shi[0] - slo[0]);
        if (!(sc > 0.f)) sc = 1.f;
        affine[brick] = make_float2(sc, off);
        slo[0] = off;
        shi[0] = sc;
    }
    __syncthreads();
    const float off = slo[0], sc = shi[0];
    for (int i = threadIdx.x; i < V; i += blockDim.x)
    {
        const float4 c = src[i];
        ushort4 q;
        q.x = __half_as_ushort(__float2half_rn((c.x - off) / sc));
        q.y = __half_as_ushort(__float2half_rn(c.y));
        q.z = __half_as_ushort(__float2half_rn(c.z));
        q.w = __half_as_ushort(__float2half_rn(c.w));
        out[brick * V + i] = q;
    }
}

} // namespace

namespace {

// Dense stencil records from the voxel payload: xpair[v] = {phin[v],
// phin[v+1]} (x neighbour clamped at the last column), cell8[v] = phi of the
// 8 cell corners (neighbours clamped at the upper faces; cells there are never
// interpolated because their upper corners are outside the grid).
__global__ void k_stencil_layouts(const float4* __restrict__ phin, int nx, int ny, int nz,
                                  float4* __restrict__ xpair, float4* __restrict__ cell8)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t N = (int64_t)nx * ny * nz;
    if (v >= N) return;
    const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((int64_t)nx * ny));
    const int64_t dx = i + 1 < nx ? 1 : 0;
    const int64_t dy = j + 1 < ny ? nx : 0;
    const int64_t dz = k + 1 < nz ? (int64_t)nx * ny : 0;
    const float4 a = phin[v];
    xpair[2 * v] = a;
    xpair[2 * v + 1] = phin[v + dx];
    cell8[2 * v] = make_float4(a.x, phin[v + dx].x, phin[v + dy].x, phin[v + dx + dy].x);
    cell8[2 * v + 1] = make_float4(phin[v + dz].x, phin[v + dx + dz].x, phin[v + dy + dz].x,
                                   phin[v + dx + dy + dz].x);
}

// Sparse stencil records, per stored voxel: neighbours are found through the
// block table; a neighbour whose block is not stored gets phi = NaN, which
// makes any query touching it invalid (as a missing block does in the
// reference); neighbours outside the grid repeat the voxel (never read).
__global__ void k_sparse_stencil_layouts(const float4* __restrict__ phin,
                                         const int32_t* __restrict__ ijk,
                                         const int32_t* __restrict__ table, int nx, int ny, int nz,
                                         int bd, int nbx, int nby, int64_t stored,
                                         float4* __restrict__ xpair, float4* __restrict__ cell8)
{
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= stored) return;
    const int V = bd * bd * bd;
    const int blk = (int)(v / V), local = (int)(v % V);
    const int i = ijk[3 * blk] * bd + local % bd;
    const int j = ijk[3 * blk + 1] * bd + (local / bd) % bd;
    const int k = ijk[3 * blk + 2] * bd + local / (bd * bd);
    const float4 self = phin[v];
    auto at = [&](int di, int dj, int dk) -> float4 {
        const int ii = i + di, jj = j + dj, kk = k + dk;
        if (ii >= nx || jj >= ny || kk >= nz) return self;
        const int b2 = table[ii / bd + nbx * (jj / bd + nby * (kk / bd))];
        if (b2 < 0) return make_float4(NAN, NAN, NAN, NAN);
        return phin[(int64_t)b2 * V + (ii % bd) + bd * ((jj % bd) + bd * (kk % bd))];
    };
    xpair[2 * v] = self;
    xpair[2 * v + 1] = at(1, 0, 0);
    if (!cell8) return;
    cell8[2 * v] = make_float4(self.x, at(1, 0, 0).x, at(0, 1, 0).x, at(1, 1, 0).x);
    cell8[2 * v + 1] = make_float4(at(0, 0, 1).x, at(1, 0, 1).x, at(0, 1, 1).x, at(1, 1, 1).x);
}

} // namespace

namespace {
// 0 automatic, 1 always, 2 never
std::atomic<int> g_sparse_pairs{0};
// Pools up to this size get pair records automatically: with the records
// (twice the pool) they stay mostly in the 126 MB L2, where one load per row
// pays (hollow cylinder 6.8 MB pool: 23.1 -> 24.4 G queries/s; 256 gears, each
// queried in turn: 15.8 -> 17.7).  A larger pool is gathered from DRAM at
// random, where the doubled footprint costs more than the saved loads (the
// 162 MB icosphere pool: 23.8 -> 20.1).
constexpr int64_t kAutoPairPoolBytes = int64_t(48) << 20;
} // namespace

int sparse_pair_records() { return g_sparse_pairs.load(); }
void set_sparse_pair_records(int mode) { g_sparse_pairs.store(mode); }

void build_stencil_layouts(sdfo_grid* g, cudaStream_t s)
{
    if (g->stored_voxels == 0 || g->info.storage != SDFO_STORAGE_FP32 || g->d.phin == nullptr)
        return;
    const int64_t N = g->stored_voxels;
    if (g->info.layout == SDFO_LAYOUT_DENSE)
    {
        if (!g->d.xpair) g->d.xpair = dalloc<float4>((size_t)N * 2);
        if (!g->d.cell8) g->d.cell8 = dalloc<float4>((size_t)N * 2);
        k_stencil_layouts<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(
            g->d.phin, g->info.shape[0], g->info.shape[1], g->info.shape[2], g->d.xpair, g->d.cell8);
    }
    else
    {
        // sparse 8^3 bricks: the x-pair records only (Tricubic rows, one
        // 256-bit load each, the +x neighbour read across the brick face)
        const int mode = sparse_pair_records();
        const bool want = mode == 1 || (mode == 0 && N * (int64_t)sizeof(float4) <= kAutoPairPoolBytes);
        if (g->info.block_dim != 8 || !want) return;
        if (!g->d.xpair) g->d.xpair = dalloc<float4>((size_t)N * 2);
        k_sparse_stencil_layouts<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(
            g->d.phin, g->d.ijk, g->d.table, g->info.shape[0], g->info.shape[1], g->info.shape[2],
            g->info.block_dim, g->nb[0], g->nb[1], N, g->d.xpair, nullptr);
    }
    SDFO_CHECK_LAUNCH();
}

void encode_fp16(const sdfo_grid* src, sdfo_grid* dst, cudaStream_t s)
{
    const int V = src->info.block_dim * src->info.block_dim * src->info.block_dim;
    const int64_t B = src->info.block_count;
    dst->d.phin16 = dalloc<ushort4>((size_t)B * V);
    dst->d.brick_affine = dalloc<float2>((size_t)B);
    if (B > 0)
    {
        k_encode_fp16<<<(unsigned)B, 256, 0, s>>>(src->d.phin, V, dst->d.phin16,
                                                    dst->d.brick_affine);
        SDFO_CHECK_LAUNCH();
    }
}

} // namespace sdfo

sdfo_grid::~sdfo_grid()
{
    using sdfo::device_free;
    sdfo::destroy_host_pipe(host_pipe);
    device_free(ws);
    // stencil records belong to the handle (views have none; the grids of a
    // batched build allocate theirs outside the shared arena)
    device_free(d.xpair);
    device_free(d.cell8);
    if (borrowed) return;
    device_free(d.phin);
    device_free(d.hess6);
    device_free(d.phi64);
    device_free(d.n64);
    device_free(d.w64);
    device_free(d.h64);
    device_free(d.table);
    device_free(d.ijk);
    device_free(d.phin16);
    device_free(d.brick_affine);
    device_free(d.ca_count);
    device_free(d.ca_phi64);
    device_free(d.ca_n64);
    device_free(d.ca_phi32);
    device_free(d.ca_n32);
    device_free(d.ca_branch);
}

using namespace sdfo;

extern "C" {

int sdfo_last_error(char* buf, size_t len)
{
    if (!buf || len == 0) return SDFO_ERR_INVALID_ARGUMENT;
    const std::string& e = last_error();
    const size_t n = e.size() < len - 1 ? e.size() : len - 1;
    std::memcpy(buf, e.data(), n);
    buf[n] = '\0';
    return SDFO_OK;
}

int sdfo_grid_create_dense(const sdfo_grid_info* info, const double* h_phi,
                           const double* h_normal, const double* h_hessian6,
                           const double* h_witness, void* stream, sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        check_spec(info);
        SDFO_REQUIRE(h_phi && h_normal, SDFO_ERR_INVALID_ARGUMENT, "phi and normal are required");
        const int64_t N = (int64_t)info->shape[0] * info->shape[1] * info->shape[2];
        std::unique_ptr<sdfo_grid> g(new sdfo_grid());
        g->info = *info;
        g->info.candidate_stride = 0;
        g->info.layout = SDFO_LAYOUT_DENSE;
        g->info.storage = SDFO_STORAGE_FP32;
        g->info.has_hessian = h_hessian6 != nullptr;
        g->info.block_dim = g->info.halo_voxels = g->info.block_count = 0;
        g->info.band_distance = 0.0;
        g->stored_voxels = N;
        SDFO_CUDA(cudaGetDevice(&g->device));
        cudaStream_t s = as_stream(stream);
        std::vector<float4> phin((size_t)N);
        for (int64_t i = 0; i < N; ++i)
            phin[(size_t)i] = make_float4((float)h_phi[i], (float)h_normal[3 * i],
                                          (float)h_normal[3 * i + 1], (float)h_normal[3 * i + 2]);
        g->d.phin = dalloc<float4>((size_t)N);
        g->d.phi64 = dalloc<double>((size_t)N);
        g->d.n64 = dalloc<double>((size_t)N * 3);
        SDFO_CUDA(cudaMemcpyAsync(g->d.phin, phin.data(), sizeof(float4) * N, cudaMemcpyHostToDevice, s));
        SDFO_CUDA(cudaMemcpyAsync(g->d.phi64, h_phi, sizeof(double) * N, cudaMemcpyHostToDevice, s));
        SDFO_CUDA(cudaMemcpyAsync(g->d.n64, h_normal, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
        std::vector<float> hs;
        if (h_hessian6)
        {
            hs.resize((size_t)N * 6);
            for (int64_t i = 0; i < N * 6; ++i) hs[(size_t)i] = (float)h_hessian6[i];
            g->d.hess6 = dalloc<float>((size_t)N * 6);
            g->d.h64 = dalloc<double>((size_t)N * 6);
            SDFO_CUDA(cudaMemcpyAsync(g->d.hess6, hs.data(), sizeof(float) * 6 * N, cudaMemcpyHostToDevice, s));
            SDFO_CUDA(cudaMemcpyAsync(g->d.h64, h_hessian6, sizeof(double) * 6 * N, cudaMemcpyHostToDevice, s));
        }
        if (h_witness)
        {
            g->d.w64 = dalloc<double>((size_t)N * 3);
            SDFO_CUDA(cudaMemcpyAsync(g->d.w64, h_witness, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
        }
        build_stencil_layouts(g.get(), s);
        SDFO_CUDA(cudaStreamSynchronize(s));
        *out = g.release();
    });
}

int sdfo_grid_create_sparse(const sdfo_grid_info* info, const int32_t* h_block_ijk,
                            const float* h_phi, const float* h_normal, const float* h_hessian6,
                            void* stream, sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "out is NULL");
        *out = nullptr;
        check_spec(info);
        const int bd = info->block_dim;
        SDFO_REQUIRE(bd > 0 && bd <= 64, SDFO_ERR_INVALID_ARGUMENT,
                     "Sparse SDF blockDim must be positive");
        const int64_t B = info->block_count;
        SDFO_REQUIRE(B >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative block count");
        SDFO_REQUIRE(B == 0 || (h_block_ijk && h_phi && h_normal), SDFO_ERR_INVALID_ARGUMENT,
                     "block ijk, phi and normal are required");
        const int V = bd * bd * bd;
        std::unique_ptr<sdfo_grid> g(new sdfo_grid());
        g->info = *info;
        g->info.candidate_stride = 0;
        g->info.layout = SDFO_LAYOUT_SPARSE;
        g->info.storage = SDFO_STORAGE_FP32;
        g->info.has_hessian = h_hessian6 != nullptr;
        for (int a = 0; a < 3; ++a) g->nb[a] = (info->shape[a] + bd - 1) / bd;
        g->stored_voxels = B * V;
        SDFO_CUDA(cudaGetDevice(&g->device));
        cudaStream_t s = as_stream(stream);
        const int64_t T = (int64_t)g->nb[0] * g->nb[1] * g->nb[2];
        std::vector<int32_t> table((size_t)T, -1);
        for (int64_t b = 0; b < B; ++b)
        {
            const int bi = h_block_ijk[3 * b], bj = h_block_ijk[3 * b + 1], bk = h_block_ijk[3 * b + 2];
            if (bi < 0 || bj < 0 || bk < 0 || bi >= g->nb[0] || bj >= g->nb[1] || bk >= g->nb[2])
                continue; // unreachable by any in-grid voxel
            int32_t& slot = table[(size_t)(bi + (int64_t)g->nb[0] * (bj + (int64_t)g->nb[1] * bk))];
            if (slot < 0) slot = (int32_t)b; // first block wins (unordered_map::emplace)
        }
        std::vector<float4> phin((size_t)(B * V));
        for (int64_t i = 0; i < B * V; ++i)
            phin[(size_t)i] = make_float4(h_phi[i], h_normal[3 * i], h_normal[3 * i + 1], h_normal[3 * i + 2]);
        g->d.table = dalloc<int32_t>((size_t)T);
        SDFO_CUDA(cudaMemcpyAsync(g->d.table, table.data(), sizeof(int32_t) * T, cudaMemcpyHostToDevice, s));
        if (B > 0)
        {
            g->d.ijk = dalloc<int32_t>((size_t)B * 3);
            g->d.phin = dalloc<float4>((size_t)(B * V));
            SDFO_CUDA(cudaMemcpyAsync(g->d.ijk, h_block_ijk, sizeof(int32_t) * 3 * B, cudaMemcpyHostToDevice, s));
            SDFO_CUDA(cudaMemcpyAsync(g->d.phin, phin.data(), sizeof(float4) * B * V, cudaMemcpyHostToDevice, s));
            if (h_hessian6)
            {
                g->d.hess6 = dalloc<float>((size_t)(B * V * 6));
                SDFO_CUDA(cudaMemcpyAsync(g->d.hess6, h_hessian6, sizeof(float) * 6 * B * V, cudaMemcpyHostToDevice, s));
            }
        }
        build_stencil_layouts(g.get(), s);
        SDFO_CUDA(cudaStreamSynchronize(s));
        *out = g.release();
    });
}

int sdfo_grid_to_fp16(const sdfo_grid* src, void* stream, sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(src && out, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = nullptr;
        SDFO_REQUIRE(src->info.layout == SDFO_LAYOUT_SPARSE && src->info.storage == SDFO_STORAGE_FP32,
                     SDFO_ERR_UNSUPPORTED, "FP16 storage is provided for sparse FP32 grids");
        cudaStream_t s = as_stream(stream);
        std::unique_ptr<sdfo_grid> g(new sdfo_grid());
        g->info = src->info;
        g->info.storage = SDFO_STORAGE_FP16;
        g->device = src->device;
        g->stored_voxels = src->stored_voxels;
        for (int a = 0; a < 3; ++a) g->nb[a] = src->nb[a];
        const int64_t T = (int64_t)g->nb[0] * g->nb[1] * g->nb[2];
        const int64_t B = src->info.block_count;
        g->d.table = dalloc<int32_t>((size_t)T);
        SDFO_CUDA(cudaMemcpyAsync(g->d.table, src->d.table, sizeof(int32_t) * T, cudaMemcpyDeviceToDevice, s));
        if (B > 0)
        {
            g->d.ijk = dalloc<int32_t>((size_t)B * 3);
            SDFO_CUDA(cudaMemcpyAsync(g->d.ijk, src->d.ijk, sizeof(int32_t) * 3 * B, cudaMemcpyDeviceToDevice, s));
        }
        if (src->d.hess6)
        {
            g->d.hess6 = dalloc<float>((size_t)src->stored_voxels * 6);
            SDFO_CUDA(cudaMemcpyAsync(g->d.hess6, src->d.hess6, sizeof(float) * 6 * src->stored_voxels,
                                      cudaMemcpyDeviceToDevice, s));
        }
        encode_fp16(src, g.get(), s);
        SDFO_CUDA(cudaStreamSynchronize(s));
        *out = g.release();
    });
}

int sdfo_grid_export_dense(const sdfo_grid* g, double* h_phi, double* h_normal,
                           double* h_hessian6, double* h_witness)
{
    return guarded([&] {
        SDFO_REQUIRE(g != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
        SDFO_REQUIRE(g->info.layout == SDFO_LAYOUT_DENSE, SDFO_ERR_INVALID_ARGUMENT,
                     "not a dense grid");
        const int64_t N = g->stored_voxels;
        std::vector<float4> phin;
        auto need_phin = [&] {
            if (phin.empty())
            {
                phin.resize((size_t)N);
                SDFO_CUDA(cudaMemcpy(phin.data(), g->d.phin, sizeof(float4) * N, cudaMemcpyDeviceToHost));
            }
        };
        if (h_phi)
        {
            if (g->d.phi64)
                SDFO_CUDA(cudaMemcpy(h_phi, g->d.phi64, sizeof(double) * N, cudaMemcpyDeviceToHost));
            else
            {
                need_phin();
                for (int64_t i = 0; i < N; ++i) h_phi[i] = phin[(size_t)i].x;
            }
        }
        if (h_normal)
        {
            if (g->d.n64)
                SDFO_CUDA(cudaMemcpy(h_normal, g->d.n64, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
            else
            {
                need_phin();
                for (int64_t i = 0; i < N; ++i)
                {
                    h_normal[3 * i] = phin[(size_t)i].y;
                    h_normal[3 * i + 1] = phin[(size_t)i].z;
                    h_normal[3 * i + 2] = phin[(size_t)i].w;
                }
            }
        }
        if (h_hessian6)
        {
            if (g->d.h64)
                SDFO_CUDA(cudaMemcpy(h_hessian6, g->d.h64, sizeof(double) * 6 * N, cudaMemcpyDeviceToHost));
            else if (g->d.hess6)
            {
                std::vector<float> hs((size_t)N * 6);
                SDFO_CUDA(cudaMemcpy(hs.data(), g->d.hess6, sizeof(float) * 6 * N, cudaMemcpyDeviceToHost));
                for (int64_t i = 0; i < N * 6; ++i) h_hessian6[i] = hs[(size_t)i];
            }
            else
                std::memset(h_hessian6, 0, sizeof(double) * 6 * N);
        }
        if (h_witness)
        {
            if (g->d.w64)
                SDFO_CUDA(cudaMemcpy(h_witness, g->d.w64, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost));
            else
                std::memset(h_witness, 0, sizeof(double) * 3 * N);
        }
    });
}

int sdfo_grid_export_sparse(const sdfo_grid* g, int32_t* h_block_ijk, float* h_phi,
                            float* h_normal, float* h_hessian6)
{
    return guarded([&] {
        SDFO_REQUIRE(g != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
        SDFO_REQUIRE(g->info.layout == SDFO_LAYOUT_SPARSE, SDFO_ERR_INVALID_ARGUMENT,
                     "not a sparse grid");
        const int64_t B = g->info.block_count;
        const int64_t N = g->stored_voxels;
        if (B == 0) return;
        if (h_block_ijk)
            SDFO_CUDA(cudaMemcpy(h_block_ijk, g->d.ijk, sizeof(int32_t) * 3 * B, cudaMemcpyDeviceToHost));
        if (h_phi || h_normal)
        {
            std::vector<float4> phin((size_t)N);
            if (g->info.storage == SDFO_STORAGE_FP16)
            {
                std::vector<ushort4> q((size_t)N);
                std::vector<float2> aff((size_t)B);
                SDFO_CUDA(cudaMemcpy(q.data(), g->d.phin16, sizeof(ushort4) * N, cudaMemcpyDeviceToHost));
                SDFO_CUDA(cudaMemcpy(aff.data(), g->d.brick_affine, sizeof(float2) * B, cudaMemcpyDeviceToHost));
                const int V = g->info.block_dim * g->info.block_dim * g->info.block_dim;
                for (int64_t i = 0; i < N; ++i)
                {
                    const float2 a = aff[(size_t)(i / V)];
                    const ushort4 v = q[(size_t)i];
                    phin[(size_t)i] = make_float4(__half2float(__ushort_as_half(v.x)) * a.x + a.y,
                                                  __half2float(__ushort_as_half(v.y)),
                                                  __half2float(__ushort_as_half(v.z)),
                                                  __half2float(__ushort_as_half(v.w)));
                }
            }
            else
            {
                SDFO_CUDA(cudaMemcpy(phin.data(), g->d.phin, sizeof(float4) * N, cudaMemcpyDeviceToHost));
            }
            for (int64_t i = 0; i < N; ++i)
            {
                if (h_phi) h_phi[i] = phin[(size_t)i].x;
                if (h_normal)
                {
                    h_normal[3 * i] = phin[(size_t)i].y;
                    h_normal[3 * i + 1] = phin[(size_t)i].z;
                    h_normal[3 * i + 2] = phin[(size_t)i].w;
                }
            }
        }
        if (h_hessian6)
        {
            if (g->d.hess6)
                SDFO_CUDA(cudaMemcpy(h_hessian6, g->d.hess6, sizeof(float) * 6 * N, cudaMemcpyDeviceToHost));
            else
                std::memset(h_hessian6, 0, sizeof(float) * 6 * N);
        }
    });
}

int sdfo_grid_get_info(const sdfo_grid* g, sdfo_grid_info* out)
{
    return guarded([&] {
        SDFO_REQUIRE(g && out, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = g->info;
    });
}

int sdfo_grid_build_stats(const sdfo_grid* g, sdfo_build_stats* out)
{
    return guarded([&] {
        SDFO_REQUIRE(g && out, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = g->stats;
    });
}

int sdfo_grid_device_views(const sdfo_grid* g, sdfo_device_views* out)
{
    return guarded([&] {
        SDFO_REQUIRE(g && out, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        std::memset(out, 0, sizeof(*out));
        out->phin = g->info.storage == SDFO_STORAGE_FP16 ? (void*)g->d.phin16 : (void*)g->d.phin;
        out->hessian6 = g->d.hess6;
        out->table = g->d.table;
        out->block_ijk = g->d.ijk;
        out->stored_voxels = g->stored_voxels;
        for (int a = 0; a < 3; ++a) out->table_dims[a] = g->nb[a];
    });
}

int sdfo_grid_copy_payload(const sdfo_grid* g, void* d_dst, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(g && d_dst, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        SDFO_REQUIRE(g->info.storage == SDFO_STORAGE_FP32, SDFO_ERR_UNSUPPORTED,
                     "payload copy needs FP32 storage");
        if (g->stored_voxels > 0)
            SDFO_CUDA(cudaMemcpyAsync(d_dst, g->d.phin, sizeof(float4) * g->stored_voxels,
                                      cudaMemcpyDeviceToDevice, as_stream(stream)));
    });
}

int sdfo_grid_export_candidates(const sdfo_grid* g, uint8_t* h_count, double* h_phi,
                                double* h_normal, int32_t* h_branch)
{
    return guarded([&] {
        SDFO_REQUIRE(g != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
        SDFO_REQUIRE(g->ca_stride > 0, SDFO_ERR_INVALID_ARGUMENT, "grid has no contact-aware candidates");
        const int64_t N = g->stored_voxels;
        const int64_t M = N * g->ca_stride;
        if (N == 0) return;
        if (h_count) SDFO_CUDA(cudaMemcpy(h_count, g->d.ca_count, (size_t)N, cudaMemcpyDeviceToHost));
        if (h_branch)
            SDFO_CUDA(cudaMemcpy(h_branch, g->d.ca_branch, sizeof(int32_t) * M, cudaMemcpyDeviceToHost));
        if (g->d.ca_phi64)
        {
            if (h_phi) SDFO_CUDA(cudaMemcpy(h_phi, g->d.ca_phi64, sizeof(double) * M, cudaMemcpyDeviceToHost));
            if (h_normal)
                SDFO_CUDA(cudaMemcpy(h_normal, g->d.ca_n64, sizeof(double) * 3 * M, cudaMemcpyDeviceToHost));
            return;
        }
        std::vector<float> tmp((size_t)(3 * M));
        if (h_phi)
        {
            SDFO_CUDA(cudaMemcpy(tmp.data(), g->d.ca_phi32, sizeof(float) * M, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < M; ++i) h_phi[i] = (double)tmp[(size_t)i];
        }
        if (h_normal)
        {
            SDFO_CUDA(cudaMemcpy(tmp.data(), g->d.ca_n32, sizeof(float) * 3 * M, cudaMemcpyDeviceToHost));
            for (int64_t i = 0; i < 3 * M; ++i) h_normal[i] = (double)tmp[(size_t)i];
        }
    });
}

int sdfo_grid_attach_candidates(sdfo_grid* g, int32_t stride, const uint8_t* h_count,
                                const double* h_phi, const double* h_normal,
                                const int32_t* h_branch)
{
    return guarded([&] {
        SDFO_REQUIRE(g && h_count && h_phi && h_normal && h_branch, SDFO_ERR_INVALID_ARGUMENT,
                     "NULL argument");
        SDFO_REQUIRE(stride >= 1 && stride <= 8, SDFO_ERR_INVALID_ARGUMENT,
                     "candidate stride must be 1..8");
        SDFO_REQUIRE(!g->borrowed && g->ca_stride == 0, SDFO_ERR_INVALID_ARGUMENT,
                     "candidates can be attached once, to an owning grid");
        const int64_t N = g->stored_voxels;
        const int64_t M = N * stride;
        if (N == 0) return;
        g->d.ca_count = dalloc<uint8_t>((size_t)N);
        g->d.ca_branch = dalloc<int32_t>((size_t)M);
        SDFO_CUDA(cudaMemcpy(g->d.ca_count, h_count, (size_t)N, cudaMemcpyHostToDevice));
        SDFO_CUDA(cudaMemcpy(g->d.ca_branch, h_branch, sizeof(int32_t) * M, cudaMemcpyHostToDevice));
        if (g->info.layout == SDFO_LAYOUT_DENSE)
        {
            g->d.ca_phi64 = dalloc<double>((size_t)M);
            g->d.ca_n64 = dalloc<double>((size_t)M * 3);
            SDFO_CUDA(cudaMemcpy(g->d.ca_phi64, h_phi, sizeof(double) * M, cudaMemcpyHostToDevice));
            SDFO_CUDA(cudaMemcpy(g->d.ca_n64, h_normal, sizeof(double) * 3 * M, cudaMemcpyHostToDevice));
        }
        else
        {
            std::vector<float> f((size_t)(3 * M));
            for (int64_t i = 0; i < M; ++i) f[(size_t)i] = (float)h_phi[i];
            g->d.ca_phi32 = dalloc<float>((size_t)M);
            SDFO_CUDA(cudaMemcpy(g->d.ca_phi32, f.data(), sizeof(float) * M, cudaMemcpyHostToDevice));
            for (int64_t i = 0; i < 3 * M; ++i) f[(size_t)i] = (float)h_normal[i];
            g->d.ca_n32 = dalloc<float>((size_t)M * 3);
            SDFO_CUDA(cudaMemcpy(g->d.ca_n32, f.data(), sizeof(float) * 3 * M, cudaMemcpyHostToDevice));
        }
        g->ca_stride = stride;
        g->info.candidate_stride = stride;
    });
}

int sdfo_grid_create_view(const sdfo_grid* g, void* d_phin, sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(g && d_phin && out, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = nullptr;
        SDFO_REQUIRE(g->info.storage == SDFO_STORAGE_FP32, SDFO_ERR_UNSUPPORTED,
                     "views need FP32 storage");
        SDFO_REQUIRE((reinterpret_cast<uintptr_t>(d_phin) & 15) == 0, SDFO_ERR_INVALID_ARGUMENT,
                     "payload must be 16-byte aligned");
        std::unique_ptr<sdfo_grid> v(new sdfo_grid());
        v->info = g->info;
        v->device = g->device;
        v->stored_voxels = g->stored_voxels;
        for (int a = 0; a < 3; ++a) v->nb[a] = g->nb[a];
        v->d = g->d;
        v->d.phin = static_cast<float4*>(d_phin);
        v->d.phi64 = v->d.n64 = v->d.w64 = v->d.h64 = nullptr; // export reads the live payload
        v->d.xpair = v->d.cell8 = nullptr; // stencil copies would go stale: read the payload
        v->borrowed = true;
        v->arena = g->arena;
        *out = v.release();
    });
}

int sdfo_grid_destroy(sdfo_grid* g)
{
    return guarded([&] { delete g; });
}

} // extern "C"
