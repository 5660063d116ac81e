// Batched sparse narrow-band build over many meshes of uneven size.
//
// Every grid is the one SdfBuilder::buildSparse (SdfBuilder.cpp:823-983)
// makes for its mesh; the batch changes how the work is scheduled, not what
// is computed (the per-block and per-voxel device functions are those of the
// single-mesh builder, in this -fmad=false translation unit):
//   host      per-mesh setupGrid and reference trees on host threads (or one
//             device LBVH per mesh), concatenated into one upload;
//   launch 1  block activation over the candidate blocks of all meshes
//             (thread -> global candidate -> mesh by binary search);
//   launch 2  one exclusive scan of the flags: the slots of each mesh are
//             contiguous and in its (bk, bj, bi) order;
//   launch 3  block table + block coordinates;
//   launch 4  persistent brick fill: about as many CTAs as fit on the 148
//             SMs, each taking the next brick of any mesh from one atomic
//             work counter, so small and large meshes share the GPU evenly;
//   launch 5  Hessian of every stored voxel.
// The grids then share one device arena (table, block coordinates, payload,
// Hessians), each handle holding a slice and a reference to the arena.
#include <atomic>
#include <exception>
#include <mutex>
#include <thread>

#include "build_common.cuh"

namespace sdfo {
namespace {

struct BatchMeta
{
    SpecD spec;
    int nb[3];
    int pad0;
    double activation;
    int64_t cand_off; // first candidate block (and table entry) of the mesh
};

template <class Tree>
__global__ void __launch_bounds__(256, SDFO_FILL_MIN_BLOCKS)
    k_batch_activate(const Tree* __restrict__ trees, const BatchMeta* __restrict__ meta,
                     const int64_t* __restrict__ cand_offs, int n, int bd, int64_t total,
                     int32_t* __restrict__ flags, int* status)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (int64_t)gridDim.x * blockDim.x)
    {
        const int m = find_segment(cand_offs, n, c);
        const BatchMeta& g = meta[m];
        flags[c] = block_active(trees[m], g.spec, bd, g.nb[0], g.nb[1], (int)(c - g.cand_off),
                                g.activation, status);
    }
}

// slot_offs[m] = first brick slot of mesh m (exclusive scan at its first
// candidate), slot_offs[n] = total bricks.
__global__ void k_batch_slot_offsets(const int64_t* __restrict__ cand_offs, int n, int64_t total,
                                     const int32_t* __restrict__ flags,
                                     const int32_t* __restrict__ slots, int64_t* __restrict__ slot_offs)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m > n) return;
    if (m == n)
        slot_offs[n] = (int64_t)slots[total - 1] + flags[total - 1];
    else
        slot_offs[m] = slots[cand_offs[m]];
}

__global__ void k_batch_table(const BatchMeta* __restrict__ meta, const int64_t* __restrict__ cand_offs,
                              const int64_t* __restrict__ slot_offs, int n, int64_t total,
                              const int32_t* __restrict__ flags, const int32_t* __restrict__ slots,
                              int32_t* __restrict__ table, int32_t* __restrict__ ijk)
{
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (int64_t)gridDim.x * blockDim.x)
    {
        const int m = find_segment(cand_offs, n, c);
        const int nbx = meta[m].nb[0], nby = meta[m].nb[1];
        const int bl = (int)(c - meta[m].cand_off);
        if (flags[c])
        {
            const int64_t slot = slots[c];
            table[c] = (int32_t)(slot - slot_offs[m]);
            ijk[3 * slot + 0] = bl % nbx;
            ijk[3 * slot + 1] = (bl / nbx) % nby;
            ijk[3 * slot + 2] = bl / (nbx * nby);
        }
        else
        {
            table[c] = -1;
        }
    }
}

// Persistent brick fill: CTAs loop taking the next brick from `next` until
// the bricks run out (the counter only grows, so every CTA ends).  Register
// budget as the single-mesh fills (SDFO_FILL_MIN_BLOCKS CTAs per SM).
template <class Tree>
__global__ void __launch_bounds__(256, SDFO_FILL_MIN_BLOCKS)
    k_batch_fill(const Tree* __restrict__ trees, const BatchMeta* __restrict__ meta,
                 const int64_t* __restrict__ slot_offs, int n, int bd, int64_t nbricks,
                 const int32_t* __restrict__ ijk, float4* __restrict__ phin,
                 unsigned long long* __restrict__ next, int* status)
{
    __shared__ long long s_brick;
    const int V = bd * bd * bd;
    for (;;)
    {
        if (threadIdx.x == 0) s_brick = (long long)atomicAdd(next, 1ull);
        __syncthreads();
        const int64_t brick = s_brick;
        __syncthreads();
        if (brick >= nbricks) break;
        const int m = find_segment(slot_offs, n, brick);
        const int bi = ijk[3 * brick], bj = ijk[3 * brick + 1], bk = ijk[3 * brick + 2];
        for (int local = threadIdx.x; local < V; local += blockDim.x)
            phin[brick * V + local] =
                brick_voxel(trees[m], meta[m].spec, bd, bi, bj, bk, local, status);
    }
}

__global__ void k_batch_hessian(const BatchMeta* __restrict__ meta,
                                const int64_t* __restrict__ slot_offs, int n, int bd,
                                int64_t stored, const int32_t* __restrict__ ijk,
                                const int32_t* __restrict__ table, const float4* __restrict__ phin,
                                float* __restrict__ hess6)
{
    const int V = bd * bd * bd;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < stored;
         v += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t brick = v / V;
        const int m = find_segment(slot_offs, n, brick);
        const BatchMeta& g = meta[m];
        const int64_t s0 = slot_offs[m];
        sparse_hessian_voxel(g.spec, bd, g.nb[0], g.nb[1], ijk + 3 * s0, table + g.cand_off,
                             phin + s0 * V, (int)(brick - s0), (int)(v % V), hess6 + 6 * v);
    }
}

// Grid size for a grid-stride launch: enough CTAs to fill every SM.
unsigned stride_blocks(int64_t work, int threads)
{
    const int sms = current_sm_count();
    const int64_t want = (work + threads - 1) / threads;
    const int64_t cap = (int64_t)sms * 16;
    return (unsigned)std::max<int64_t>(1, std::min(want, cap));
}

std::atomic<int> g_fill_ctas_per_sm{0};

// Device storage of all grids of the batch, freed with the last handle.
struct Arena
{
    void* base = nullptr;
    ~Arena() { device_free(base); }
};

template <class T>
T* carve(unsigned char*& p, size_t count)
{
    T* r = reinterpret_cast<T*>(p);
    p += (count * sizeof(T) + 255) & ~size_t(255);
    return r;
}

} // namespace

void set_fill_ctas_per_sm(int k) { g_fill_ctas_per_sm.store(k); }
int fill_ctas_per_sm() { return g_fill_ctas_per_sm.load(); }

std::vector<sdfo_grid*> build_sparse_batched(const sdfo_mesh_desc* meshes, int n, cudaStream_t s)
{
    const auto t0 = std::chrono::steady_clock::now();
    const int bd = meshes[0].params.block_dim;
    const int V = bd * bd * bd;
    std::vector<sdfo_grid_info> info((size_t)n);
    std::vector<BatchMeta> meta((size_t)n);
    std::vector<int64_t> cand_offs((size_t)n + 1, 0);
    bool any_hessian = false;
    for (int m = 0; m < n; ++m)
    {
        const sdfo_mesh_desc& d = meshes[m];
        const sdfo_sparse_build_params& p = d.params;
        SDFO_REQUIRE(p.block_dim == bd, SDFO_ERR_INVALID_ARGUMENT,
                     "all meshes of a batched build must use the same blockDim");
        sdfo_grid_info gi = setup_grid(d.h_verts, d.nv, p.base);
        // SdfBuilder.cpp:835-842, as in the single-mesh builder
        const double h = std::max({gi.voxel[0], gi.voxel[1], gi.voxel[2]});
        const double band = p.band_distance > 0.0 ? p.band_distance : (double)p.band_voxels * h;
        const double blockRadius = 0.5 * std::sqrt(3.0) * (double)bd * h;
        volatile double act = band + (double)p.halo_voxels * h;
        act = act + blockRadius;
        gi.layout = SDFO_LAYOUT_SPARSE;
        gi.block_dim = bd;
        gi.halo_voxels = p.halo_voxels;
        gi.band_distance = band;
        gi.has_hessian = p.store_hessian ? 1 : 0;
        any_hessian = any_hessian || p.store_hessian;
        BatchMeta& bm = meta[(size_t)m];
        bm.spec = spec_of(gi);
        bm.activation = act;
        int64_t cand = 1;
        for (int a = 0; a < 3; ++a)
        {
            bm.nb[a] = (gi.shape[a] + bd - 1) / bd;
            cand *= bm.nb[a];
        }
        bm.cand_off = cand_offs[(size_t)m];
        cand_offs[(size_t)m + 1] = cand_offs[(size_t)m] + cand;
        info[(size_t)m] = gi;
    }
    const int64_t total = cand_offs[(size_t)n];
    SDFO_REQUIRE(total < (int64_t(1) << 31), SDFO_ERR_INVALID_ARGUMENT,
                 "batched build: more than 2^31 candidate blocks");
    const double setup_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    Timer tm(s);
    const int mode = bvh_mode();
    // trees: reference trees built on host threads and uploaded as one
    // concatenation, or one device LBVH per mesh
    DeviceBuffer<RefNode> ref_nodes;
    DeviceBuffer<double> ref_tri9;
    DeviceBuffer<float4> ref_tbox;
    DeviceBuffer<double> ref_pn; // pseudo-normal sign mode only
    const bool pseudo = sign_mode() == SDFO_SIGN_PSEUDONORMAL;
    DeviceBuffer<int32_t> ref_tri_id;
    std::vector<std::unique_ptr<DeviceLbvh>> lbvh;
    std::vector<RefTreeView> ref_views;
    std::vector<LbvhView> lbvh_views;
    int64_t total_nodes = 0;
    if (mode == SDFO_BVH_REFERENCE)
    {
        std::vector<HostTreeData> host((size_t)n);
        std::atomic<int> next{0};
        const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), (unsigned)n));
        std::vector<std::thread> pool;
        std::exception_ptr err;
        std::mutex err_mu;
        for (unsigned t = 0; t < nt; ++t)
            pool.emplace_back([&] {
                for (int m = next++; m < n; m = next++)
                {
                    try
                    {
                        // one host thread per mesh: the pool runs the meshes side by side
                        host_ref_tree(host[(size_t)m], meshes[m].h_verts, meshes[m].h_tris,
                                      meshes[m].nt, 1, false);
                    }
                    catch (...)
                    {
                        std::lock_guard<std::mutex> lk(err_mu);
                        err = std::current_exception();
                    }
                }
            });
        for (auto& th : pool) th.join();
        if (err) std::rethrow_exception(err);
        std::vector<int64_t> node_off((size_t)n + 1, 0), tri_off((size_t)n + 1, 0);
        for (int m = 0; m < n; ++m)
        {
            node_off[(size_t)m + 1] = node_off[(size_t)m] + (int64_t)host[(size_t)m].nodes.size();
            tri_off[(size_t)m + 1] = tri_off[(size_t)m] + (int64_t)host[(size_t)m].tri_id.size();
        }
        total_nodes = node_off[(size_t)n];
        std::vector<RefNode> nodes((size_t)total_nodes);
        std::vector<int32_t> tri_id((size_t)tri_off[(size_t)n]);
        std::vector<int64_t> vert_off((size_t)n + 1, 0);
        for (int m = 0; m < n; ++m)
        {
            const HostTreeData& h = host[(size_t)m];
            std::copy(h.nodes.begin(), h.nodes.end(), nodes.begin() + node_off[(size_t)m]);
            std::copy(h.tri_id.begin(), h.tri_id.end(), tri_id.begin() + tri_off[(size_t)m]);
            vert_off[(size_t)m + 1] = vert_off[(size_t)m] + meshes[m].nv;
        }
        ref_nodes.reset(nodes.size());
        ref_tri9.reset((size_t)tri_off[(size_t)n] * 9);
        ref_tbox.reset((size_t)tri_off[(size_t)n] * 2);
        ref_tri_id.reset(tri_id.size());
        SDFO_CUDA(cudaMemcpyAsync(ref_nodes.get(), nodes.data(), sizeof(RefNode) * nodes.size(),
                                  cudaMemcpyHostToDevice, s));
        SDFO_CUDA(cudaMemcpyAsync(ref_tri_id.get(), tri_id.data(), sizeof(int32_t) * tri_id.size(),
                                  cudaMemcpyHostToDevice, s));
        // the triangles in slot order are gathered on the device from each
        // mesh's vertices and (mesh-local) triangles
        DeviceBuffer<double> dverts((size_t)vert_off[(size_t)n] * 3);
        DeviceBuffer<int32_t> dtris((size_t)tri_off[(size_t)n] * 3);
        for (int m = 0; m < n; ++m)
        {
            SDFO_CUDA(cudaMemcpyAsync(dverts.get() + 3 * vert_off[(size_t)m], meshes[m].h_verts,
                                      sizeof(double) * 3 * (size_t)meshes[m].nv, cudaMemcpyHostToDevice, s));
            SDFO_CUDA(cudaMemcpyAsync(dtris.get() + 3 * tri_off[(size_t)m], meshes[m].h_tris,
                                      sizeof(int32_t) * 3 * (size_t)meshes[m].nt, cudaMemcpyHostToDevice, s));
        }
        for (int m = 0; m < n; ++m)
        {
            const int64_t nt_m = meshes[m].nt;
            if (nt_m <= 0) continue;
            k_gather_tri9<<<(unsigned)((nt_m + 255) / 256), 256, 0, s>>>(
                dverts.get() + 3 * vert_off[(size_t)m], dtris.get() + 3 * tri_off[(size_t)m],
                ref_tri_id.get() + tri_off[(size_t)m], (int)nt_m, ref_tri9.get() + 9 * tri_off[(size_t)m]);
            SDFO_CHECK_LAUNCH();
            k_tri_boxes<<<(unsigned)((nt_m + 255) / 256), 256, 0, s>>>(
                ref_tri9.get() + 9 * tri_off[(size_t)m], (int)nt_m, ref_tbox.get() + 2 * tri_off[(size_t)m]);
            SDFO_CHECK_LAUNCH();
        }
        ref_views.resize((size_t)n);
        for (int m = 0; m < n; ++m)
        {
            RefTreeView& v = ref_views[(size_t)m];
            v.nodes = ref_nodes.get() + node_off[(size_t)m];
            v.tri9 = ref_tri9.get() + 9 * tri_off[(size_t)m];
            v.tri_id = ref_tri_id.get() + tri_off[(size_t)m];
            v.n = (int)meshes[m].nt;
            v.nnodes = (int)host[(size_t)m].nodes.size();
            parity_ray(v.dir);
            v.tbox = triangle_cull() ? ref_tbox.get() + 2 * tri_off[(size_t)m] : nullptr;
            set_cull_margins(v, scene_extent(meshes[m].h_verts, meshes[m].nv, info[(size_t)m]));
        }
        if (pseudo)
        {
            ref_pn.reset((size_t)tri_off[(size_t)n] * 18);
            for (int m = 0; m < n; ++m)
            {
                if (meshes[m].nt <= 0) continue;
                DeviceBuffer<double> one;
                upload_pseudo_normals(one, meshes[m].h_verts, meshes[m].nv, meshes[m].h_tris, meshes[m].nt,
                                      ref_tri_id.get() + tri_off[(size_t)m], s);
                SDFO_CUDA(cudaMemcpyAsync(ref_pn.get() + 18 * tri_off[(size_t)m], one.get(),
                                          sizeof(double) * 18 * (size_t)meshes[m].nt, cudaMemcpyDeviceToDevice, s));
                SDFO_CUDA(cudaStreamSynchronize(s));
                ref_views[(size_t)m].pn = ref_pn.get() + 18 * tri_off[(size_t)m];
            }
        }
        // the host vectors are freed on return from this block
        SDFO_CUDA(cudaStreamSynchronize(s));
    }
    else
    {
        lbvh.resize((size_t)n);
        lbvh_views.resize((size_t)n);
        for (int m = 0; m < n; ++m)
        {
            lbvh[(size_t)m].reset(new DeviceLbvh());
            build_lbvh(*lbvh[(size_t)m], meshes[m].h_verts, meshes[m].nv, meshes[m].h_tris,
                       meshes[m].nt, scene_extent(meshes[m].h_verts, meshes[m].nv, info[(size_t)m]), s);
            if (pseudo)
                upload_pseudo_normals(lbvh[(size_t)m]->pn, meshes[m].h_verts, meshes[m].nv, meshes[m].h_tris,
                                      meshes[m].nt, lbvh[(size_t)m]->tri_id.get(), s);
            lbvh_views[(size_t)m] = lbvh[(size_t)m]->view();
            total_nodes += meshes[m].nt > 1 ? meshes[m].nt - 1 : 0;
        }
    }
    DeviceBuffer<RefTreeView> d_ref_views(mode == SDFO_BVH_REFERENCE ? (size_t)n : 0);
    DeviceBuffer<LbvhView> d_lbvh_views(mode == SDFO_BVH_REFERENCE ? 0 : (size_t)n);
    DeviceBuffer<BatchMeta> d_meta((size_t)n);
    DeviceBuffer<int64_t> d_cand_offs((size_t)n + 1), d_slot_offs((size_t)n + 1);
    if (mode == SDFO_BVH_REFERENCE)
        SDFO_CUDA(cudaMemcpyAsync(d_ref_views.get(), ref_views.data(), sizeof(RefTreeView) * n,
                                  cudaMemcpyHostToDevice, s));
    else
        SDFO_CUDA(cudaMemcpyAsync(d_lbvh_views.get(), lbvh_views.data(), sizeof(LbvhView) * n,
                                  cudaMemcpyHostToDevice, s));
    SDFO_CUDA(cudaMemcpyAsync(d_meta.get(), meta.data(), sizeof(BatchMeta) * n,
                              cudaMemcpyHostToDevice, s));
    SDFO_CUDA(cudaMemcpyAsync(d_cand_offs.get(), cand_offs.data(), sizeof(int64_t) * (n + 1),
                              cudaMemcpyHostToDevice, s));
    const double bvh_ms = tm.lap();

    DeviceBuffer<int> status(1);
    SDFO_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), s));
    DeviceBuffer<int32_t> flags((size_t)total), slots((size_t)total);
    const int T = 256;
    if (mode == SDFO_BVH_REFERENCE)
        k_batch_activate<<<stride_blocks(total, T), T, 0, s>>>(d_ref_views.get(), d_meta.get(),
                                                               d_cand_offs.get(), n, bd, total,
                                                               flags.get(), status.get());
    else
        k_batch_activate<<<stride_blocks(total, T), T, 0, s>>>(d_lbvh_views.get(), d_meta.get(),
                                                               d_cand_offs.get(), n, bd, total,
                                                               flags.get(), status.get());
    SDFO_CHECK_LAUNCH();
    size_t temp = 0;
    SDFO_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, flags.get(), slots.get(), (int)total, s));
    DeviceBuffer<unsigned char> tmp(temp);
    SDFO_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), temp, flags.get(), slots.get(), (int)total, s));
    k_batch_slot_offsets<<<(n + 1 + T - 1) / T, T, 0, s>>>(d_cand_offs.get(), n, total, flags.get(),
                                                           slots.get(), d_slot_offs.get());
    SDFO_CHECK_LAUNCH();
    std::vector<int64_t> slot_offs((size_t)n + 1);
    SDFO_CUDA(cudaMemcpyAsync(slot_offs.data(), d_slot_offs.get(), sizeof(int64_t) * (n + 1),
                              cudaMemcpyDeviceToHost, s));
    SDFO_CUDA(cudaStreamSynchronize(s));
    const int64_t B = slot_offs[(size_t)n];
    const int64_t stored = B * V;

    // one arena: table | block coordinates | payload | Hessians
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t bytes = up(sizeof(int32_t) * (size_t)total) + up(sizeof(int32_t) * 3 * (size_t)std::max<int64_t>(B, 1)) +
                         up(sizeof(float4) * (size_t)std::max<int64_t>(stored, 1)) +
                         (any_hessian ? up(sizeof(float) * 6 * (size_t)std::max<int64_t>(stored, 1)) : 0);
    auto arena = std::make_shared<Arena>();
    arena->base = device_alloc(bytes);
    unsigned char* p = static_cast<unsigned char*>(arena->base);
    int32_t* table = carve<int32_t>(p, (size_t)total);
    int32_t* ijk = carve<int32_t>(p, 3 * (size_t)std::max<int64_t>(B, 1));
    float4* phin = carve<float4>(p, (size_t)std::max<int64_t>(stored, 1));
    float* hess6 = any_hessian ? carve<float>(p, 6 * (size_t)std::max<int64_t>(stored, 1)) : nullptr;
    k_batch_table<<<stride_blocks(total, T), T, 0, s>>>(d_meta.get(), d_cand_offs.get(),
                                                        d_slot_offs.get(), n, total, flags.get(),
                                                        slots.get(), table, ijk);
    SDFO_CHECK_LAUNCH();
    if (B > 0)
    {
        DeviceBuffer<unsigned long long> counter(1);
        SDFO_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(unsigned long long), s));
        const int sms = current_sm_count();
        int per_sm = 1;
        if (mode == SDFO_BVH_REFERENCE)
        {
            SDFO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_batch_fill<RefTreeView>, T, 0));
            if (g_fill_ctas_per_sm.load() > 0) per_sm = std::min(per_sm, g_fill_ctas_per_sm.load());
            const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(B, (int64_t)sms * std::max(per_sm, 1)));
            k_batch_fill<<<grid, T, 0, s>>>(d_ref_views.get(), d_meta.get(), d_slot_offs.get(), n, bd,
                                            B, ijk, phin, counter.get(), status.get());
        }
        else
        {
            SDFO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &per_sm, k_batch_fill<LbvhView>, T, 0));
            if (g_fill_ctas_per_sm.load() > 0) per_sm = std::min(per_sm, g_fill_ctas_per_sm.load());
            const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(B, (int64_t)sms * std::max(per_sm, 1)));
            k_batch_fill<<<grid, T, 0, s>>>(d_lbvh_views.get(), d_meta.get(), d_slot_offs.get(), n,
                                            bd, B, ijk, phin, counter.get(), status.get());
        }
        SDFO_CHECK_LAUNCH();
    }
    const double fill_ms = tm.lap();
    if (B > 0 && any_hessian)
    {
        k_batch_hessian<<<stride_blocks(stored, T), T, 0, s>>>(d_meta.get(), d_slot_offs.get(), n, bd,
                                                               stored, ijk, table, phin, hess6);
        SDFO_CHECK_LAUNCH();
    }
    const double hessian_ms = tm.lap();
    check_status(status, s);
    const double total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();

    std::vector<sdfo_grid*> out;
    out.reserve((size_t)n);
    try
    {
        int dev = 0;
        SDFO_CUDA(cudaGetDevice(&dev));
        for (int m = 0; m < n; ++m)
        {
            std::unique_ptr<sdfo_grid> g(new sdfo_grid());
            const int64_t s0 = slot_offs[(size_t)m], Bm = slot_offs[(size_t)m + 1] - s0;
            g->info = info[(size_t)m];
            g->info.block_count = (int32_t)Bm;
            g->device = dev;
            for (int a = 0; a < 3; ++a) g->nb[a] = meta[(size_t)m].nb[a];
            g->stored_voxels = Bm * V;
            g->d.table = table + cand_offs[(size_t)m];
            g->d.ijk = ijk + 3 * s0;
            g->d.phin = phin + s0 * V;
            g->d.hess6 = (hess6 && meshes[m].params.store_hessian) ? hess6 + 6 * s0 * V : nullptr;
            g->borrowed = true;
            g->arena = arena;
            g->stats.setup_ms = setup_ms;
            g->stats.bvh_ms = bvh_ms;
            g->stats.fill_ms = fill_ms;
            g->stats.hessian_ms = hessian_ms;
            g->stats.total_ms = total_ms;
            g->stats.voxels_filled = Bm * V;
            g->stats.candidate_blocks = cand_offs[(size_t)m + 1] - cand_offs[(size_t)m];
            g->stats.triangles = (int32_t)meshes[m].nt;
            g->stats.bvh_nodes = mode == SDFO_BVH_REFERENCE ? ref_views[(size_t)m].nnodes
                                                            : (int32_t)(meshes[m].nt > 1 ? meshes[m].nt - 1 : 0);
            build_stencil_layouts(g.get(), s);
            out.push_back(g.release());
        }
        SDFO_CUDA(cudaStreamSynchronize(s));
    }
    catch (...)
    {
        for (sdfo_grid* g : out) delete g;
        throw;
    }
    return out;
}

} // namespace sdfo
