// Batched queries over many grids in one launch (the multi-mesh query of
// the gear workload).  The queries of grid g form tiles of THREADS queries;
// tile k's record holds its first query, its grid and its query count.  The
// kernel is persistent and walks runs of m consecutive tiles in grid-stride
// order (CTA c takes tiles cm .. cm + m - 1, then (c + G) m .., ...), so at
// any moment the resident CTAs work on a window of consecutive tiles -- a
// few grids -- and those grids' brick pools stay in L2.  Each thread holds
// the next tile's record and point in registers before it evaluates the
// current tile (the record of the tile after that is in flight), and the
// grid descriptor and pose are read through L1 (the same few hundred bytes
// for the whole tile), so warps never wait on one another.  A query point is
// mapped into the grid's frame with the grid's rigid pose (FP64), evaluated
// with the single-grid interpolants, and its gradient rotated back to the
// world frame.  No reference counterpart: the reference queries one
// SdfOracle at a time.
#include "interp.cuh"

#include <algorithm>
#include <mutex>

namespace sdfo {
// One tile of a query batch (16 bytes, one vector load)
struct __align__(16) BatchTile
{
    int64_t q0;    // first query of the tile
    int32_t grid;  // grid of the tile
    int32_t count; // queries in the tile (1..THREADS)
};
} // namespace sdfo

struct sdfo_query_batch
{
    int n = 0;
    int device = 0;
    // launch shape: 128 threads per CTA, runs of 4 tiles (the fastest
    // measured on the 256-gear batch: 27 G queries/s against 22 for 256 x 1)
    int threads = 128;
    int run_log2 = 2; // consecutive tiles a CTA takes before it strides
    int64_t total = 0;
    sdfo::DeviceBuffer<sdfo::GridView> views;
    // tile records for 128, 256 and 512 threads per CTA
    sdfo::DeviceBuffer<sdfo::BatchTile> tiles[3];
    int64_t ntiles[3] = {0, 0, 0};
    // layouts of the grids: 0 all dense, 1 all sparse 8^3 bricks over FP32
    // pools, 4 all sparse 8^3 bricks over FP16 pools, 2 all other sparse, 3
    // mixed (the kernel is specialised on it)
    int kind = 3;
};

namespace sdfo {
namespace {

int shape_index(int threads) { return threads == 128 ? 0 : (threads == 256 ? 1 : 2); }

// Resident CTAs per SM the launch shapes ask the register allocator for:
// 128 threads, 6 CTAs (24 warps, up to 80 registers, no spills in the sparse
// Tricubic kernel); 256 and 512 threads, 32 warps (64 registers).  The shape
// is a tuning knob (sdfo_query_batch_set_threads).
template <int THREADS>
constexpr int batch_min_blocks() { return THREADS == 128 ? 6 : 1024 / THREADS; }

__device__ __forceinline__ BatchTile load_tile(const BatchTile* __restrict__ tiles, int64_t t, int64_t ntiles)
{
    BatchTile r;
    if (t < ntiles)
    {
        const int4 v = __ldg(reinterpret_cast<const int4*>(tiles + t));
        r.q0 = (int64_t)(((uint64_t)(uint32_t)v.y << 32) | (uint32_t)v.x);
        r.grid = v.z;
        r.count = v.w;
    }
    else
    {
        r.q0 = 0;
        r.grid = -1;
        r.count = 0;
    }
    return r;
}

template <int KIND, int MODE>
__device__ __forceinline__ bool evaluate_kind(const GridView& v, const double p[3], Interp& r, float unit[3])
{
    if constexpr (KIND == 0) return evaluate<MODE, false, 0, false>(v, p, r, unit);
    else if constexpr (KIND == 1) return evaluate<MODE, true, 8, false, 1>(v, p, r, unit);
    else if constexpr (KIND == 4) return evaluate<MODE, true, 8, false, 2>(v, p, r, unit);
    else if constexpr (KIND == 2) return evaluate<MODE, true, 0, false>(v, p, r, unit);
    else
    {
        if (v.layout == SDFO_LAYOUT_DENSE) return evaluate<MODE, false, 0, false>(v, p, r, unit);
        if (v.bd == 8) return evaluate<MODE, true, 8, false>(v, p, r, unit);
        return evaluate<MODE, true, 0, false>(v, p, r, unit);
    }
}

template <int MODE, int THREADS, int KIND>
__global__ void __launch_bounds__(THREADS, batch_min_blocks<THREADS>())
    k_query_batch(const GridView* __restrict__ views, const BatchTile* __restrict__ tiles, int64_t ntiles,
                  int run_log2, const sdfo_pose* __restrict__ poses, const float* __restrict__ pts,
                  float* __restrict__ gap, float* __restrict__ grad, uint8_t* __restrict__ valid)
{
    const int tid = threadIdx.x;
    const int64_t run_mask = (int64_t(1) << run_log2) - 1;
    const int64_t stride = ((int64_t)gridDim.x - 1) << run_log2;
    // the tile after t in this CTA's sequence
    auto next = [&](int64_t t) { return ((t + 1) & run_mask) ? t + 1 : t + 1 + stride; };
    int64_t t = (int64_t)blockIdx.x << run_log2;
    BatchTile cur = load_tile(tiles, t, ntiles);
    float x[3] = {0.f, 0.f, 0.f};
    if (tid < cur.count)
        for (int a = 0; a < 3; ++a) x[a] = __ldcs(pts + 3 * (cur.q0 + tid) + a);
    int64_t tn = next(t);
    BatchTile nxt = load_tile(tiles, tn, ntiles);
    for (; t < ntiles; t = tn, tn = next(tn))
    {
        // the next tile's point, the record of the tile after it
        float xn[3] = {0.f, 0.f, 0.f};
        if (tid < nxt.count)
            for (int a = 0; a < 3; ++a) xn[a] = __ldcs(pts + 3 * (nxt.q0 + tid) + a);
        const BatchTile after = load_tile(tiles, next(tn), ntiles);
        if (tid < cur.count)
        {
            const int64_t q = cur.q0 + tid;
            const GridView& v = views[cur.grid];
            double R[9], tr[3];
            if (poses)
            {
                const sdfo_pose& ps = poses[cur.grid];
                for (int a = 0; a < 9; ++a) R[a] = __ldg(ps.R + a);
                for (int a = 0; a < 3; ++a) tr[a] = __ldg(ps.t + a);
            }
            else
            {
                for (int a = 0; a < 9; ++a) R[a] = (a % 4) == 0 ? 1.0 : 0.0;
                for (int a = 0; a < 3; ++a) tr[a] = 0.0;
            }
            const double w[3] = {(double)x[0] - tr[0], (double)x[1] - tr[1], (double)x[2] - tr[2]};
            // p = R^T (x - t)
            const double p[3] = {R[0] * w[0] + R[3] * w[1] + R[6] * w[2],
                                 R[1] * w[0] + R[4] * w[1] + R[7] * w[2],
                                 R[2] * w[0] + R[5] * w[1] + R[8] * w[2]};
            Interp r;
            float unit[3];
            const bool ok = evaluate_kind<KIND, MODE>(v, p, r, unit);
            if (!ok)
            {
                r.gap = 0.f;
                r.g[0] = r.g[1] = r.g[2] = 0.f;
            }
            __stcs(gap + q, r.gap);
            if (grad)
            {
                // world gradient R g (the rotation is read again: L1 hits)
                const double* Rg = poses ? poses[cur.grid].R : nullptr;
                float gw[3];
                for (int a = 0; a < 3; ++a)
                    gw[a] = Rg ? (float)(__ldg(Rg + 3 * a) * r.g[0] + __ldg(Rg + 3 * a + 1) * r.g[1] +
                                         __ldg(Rg + 3 * a + 2) * r.g[2])
                               : r.g[a];
                for (int a = 0; a < 3; ++a) __stcs(grad + 3 * q + a, gw[a]);
            }
            if (valid) valid[q] = ok ? 1 : 0;
        }
        cur = nxt;
        nxt = after;
        for (int a = 0; a < 3; ++a) x[a] = xn[a];
    }
}

// Resident CTAs per SM of k_query_batch<MODE, THREADS, KIND> on the current device
template <int MODE, int THREADS, int KIND>
int batch_blocks_per_sm()
{
    static std::mutex mu;
    static int cached[64] = {0};
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    int& c = cached[dev & 63];
    if (c == 0)
    {
        int b = 0;
        SDFO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_query_batch<MODE, THREADS, KIND>, THREADS, 0));
        c = b > 0 ? b : 1;
    }
    return c;
}

template <int MODE, int THREADS, int KIND>
void launch_batch3(const sdfo_query_batch* b, int64_t ntiles, const BatchTile* t, const float* pts,
                   const sdfo_pose* poses, float* gap, float* grad, uint8_t* valid, cudaStream_t s)
{
    const int64_t resident = (int64_t)current_sm_count() * batch_blocks_per_sm<MODE, THREADS, KIND>();
    const int64_t runs = (ntiles + (int64_t(1) << b->run_log2) - 1) >> b->run_log2;
    const unsigned blocks = (unsigned)std::min<int64_t>(runs, resident);
    k_query_batch<MODE, THREADS, KIND><<<blocks, THREADS, 0, s>>>(b->views.get(), t, ntiles, b->run_log2,
                                                                  poses, pts, gap, grad, valid);
}

template <int MODE, int THREADS>
void launch_batch2(const sdfo_query_batch* b, int64_t ntiles, const BatchTile* t, const float* pts,
                   const sdfo_pose* poses, float* gap, float* grad, uint8_t* valid, cudaStream_t s)
{
    switch (b->kind)
    {
    case 0: launch_batch3<MODE, THREADS, 0>(b, ntiles, t, pts, poses, gap, grad, valid, s); break;
    case 1: launch_batch3<MODE, THREADS, 1>(b, ntiles, t, pts, poses, gap, grad, valid, s); break;
    case 2: launch_batch3<MODE, THREADS, 2>(b, ntiles, t, pts, poses, gap, grad, valid, s); break;
    case 4: launch_batch3<MODE, THREADS, 4>(b, ntiles, t, pts, poses, gap, grad, valid, s); break;
    default: launch_batch3<MODE, THREADS, 3>(b, ntiles, t, pts, poses, gap, grad, valid, s);
    }
}

template <int MODE>
void launch_batch(const sdfo_query_batch* b, const float* pts, const sdfo_pose* poses, float* gap,
                  float* grad, uint8_t* valid, cudaStream_t s)
{
    const int si = shape_index(b->threads);
    const int64_t ntiles = b->ntiles[si];
    if (ntiles == 0) return;
    const BatchTile* t = b->tiles[si].get();
    switch (b->threads)
    {
    case 256: launch_batch2<MODE, 256>(b, ntiles, t, pts, poses, gap, grad, valid, s); break;
    case 512: launch_batch2<MODE, 512>(b, ntiles, t, pts, poses, gap, grad, valid, s); break;
    default: launch_batch2<MODE, 128>(b, ntiles, t, pts, poses, gap, grad, valid, s);
    }
    SDFO_CHECK_LAUNCH();
}

} // namespace
} // namespace sdfo

using namespace sdfo;

extern "C" {

int sdfo_query_batch_create(const sdfo_grid* const* grids, int32_t n, const int64_t* h_counts,
                            sdfo_query_batch** out)
{
    return guarded([&] {
        SDFO_REQUIRE(out && grids && h_counts, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        *out = nullptr;
        SDFO_REQUIRE(n > 0, SDFO_ERR_INVALID_ARGUMENT, "query batch needs at least one grid");
        std::unique_ptr<sdfo_query_batch> b(new sdfo_query_batch());
        b->n = n;
        std::vector<GridView> views((size_t)n);
        int64_t total = 0, ntiles128 = 0;
        for (int g = 0; g < n; ++g)
        {
            SDFO_REQUIRE(grids[g] != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
            SDFO_REQUIRE(h_counts[g] >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
            SDFO_REQUIRE(g == 0 || grids[g]->device == grids[0]->device, SDFO_ERR_INVALID_ARGUMENT,
                         "grids of a query batch must be on one device");
            views[(size_t)g] = make_view(grids[g]);
            total += h_counts[g];
            ntiles128 += (h_counts[g] + 127) / 128;
        }
        SDFO_REQUIRE(ntiles128 < (int64_t(1) << 31), SDFO_ERR_INVALID_ARGUMENT, "too many queries in one batch");
        b->device = grids[0]->device;
        auto kind_of = [](const GridView& v) {
            if (v.layout == SDFO_LAYOUT_DENSE) return 0;
            if (v.bd != 8) return 2;
            return v.storage == SDFO_STORAGE_FP16 ? 4 : 1;
        };
        b->kind = kind_of(views[0]);
        for (int g = 1; g < n; ++g)
            if (kind_of(views[(size_t)g]) != b->kind) b->kind = 3;
        b->total = total;
        b->views.reset((size_t)n);
        SDFO_CUDA(cudaMemcpy(b->views.get(), views.data(), sizeof(GridView) * n, cudaMemcpyHostToDevice));
        const int shapes[3] = {128, 256, 512};
        for (int k = 0; k < 3; ++k)
        {
            std::vector<BatchTile> recs;
            recs.reserve((size_t)(total / shapes[k] + n));
            int64_t q0 = 0;
            for (int g = 0; g < n; ++g)
            {
                for (int64_t i = 0; i < h_counts[g]; i += shapes[k])
                    recs.push_back(BatchTile{q0 + i, g, (int32_t)std::min<int64_t>(shapes[k], h_counts[g] - i)});
                q0 += h_counts[g];
            }
            b->ntiles[k] = (int64_t)recs.size();
            if (recs.empty()) continue;
            b->tiles[k].reset(recs.size());
            SDFO_CUDA(cudaMemcpy(b->tiles[k].get(), recs.data(), sizeof(BatchTile) * recs.size(),
                                 cudaMemcpyHostToDevice));
        }
        *out = b.release();
    });
}

int sdfo_query_batch_run(const sdfo_query_batch* b, int32_t mode, const float* d_points,
                         const sdfo_pose* d_poses, float* d_gap, float* d_grad, uint8_t* d_valid,
                         void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(b != nullptr, SDFO_ERR_INVALID_ARGUMENT, "batch is NULL");
        if (b->total == 0) return;
        SDFO_REQUIRE(d_points && d_gap, SDFO_ERR_INVALID_ARGUMENT, "points and gap are required");
        cudaStream_t s = as_stream(stream);
        if (mode == SDFO_TRICUBIC)
            launch_batch<SDFO_TRICUBIC>(b, d_points, d_poses, d_gap, d_grad, d_valid, s);
        else if (mode == SDFO_TRILINEAR)
            launch_batch<SDFO_TRILINEAR>(b, d_points, d_poses, d_gap, d_grad, d_valid, s);
        else
            throw Error(SDFO_ERR_UNSUPPORTED, "batched queries support Trilinear and Tricubic");
    });
}

int sdfo_query_batch_set_threads(sdfo_query_batch* b, int32_t threads)
{
    return guarded([&] {
        SDFO_REQUIRE(b != nullptr, SDFO_ERR_INVALID_ARGUMENT, "batch is NULL");
        SDFO_REQUIRE(threads == 128 || threads == 256 || threads == 512, SDFO_ERR_INVALID_ARGUMENT,
                     "threads per CTA must be 128, 256 or 512");
        b->threads = threads;
    });
}

int sdfo_query_batch_set_run(sdfo_query_batch* b, int32_t tiles)
{
    return guarded([&] {
        SDFO_REQUIRE(b != nullptr, SDFO_ERR_INVALID_ARGUMENT, "batch is NULL");
        SDFO_REQUIRE(tiles >= 1 && tiles <= 64 && (tiles & (tiles - 1)) == 0, SDFO_ERR_INVALID_ARGUMENT,
                     "run length must be a power of two in [1, 64]");
        int k = 0;
        while ((1 << k) < tiles) ++k;
        b->run_log2 = k;
    });
}

int sdfo_query_batch_total(const sdfo_query_batch* b, int64_t* total)
{
    return guarded([&] {
        SDFO_REQUIRE(b && total, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        *total = b->total;
    });
}

int sdfo_query_batch_destroy(sdfo_query_batch* b)
{
    return guarded([&] { delete b; });
}

} // extern "C"
