// Batched queries over many grids in one launch (the multi-mesh query of
// the gear workload): CTA t of the launch takes the t-th tile of THREADS
// queries, the tile's grid found by binary search over the per-grid tile
// offsets; the grid descriptor is copied to shared memory once per CTA.  A
// query point is mapped into the grid's frame with the grid's rigid pose
// (FP64), evaluated with the single-grid interpolants, and its gradient
// rotated back to the world frame.  No reference counterpart: the reference
// queries one SdfOracle at a time.
#include "interp.cuh"

struct sdfo_query_batch
{
    int n = 0;
    int device = 0;
    int threads = 256;
    int64_t total = 0;
    sdfo::DeviceBuffer<sdfo::GridView> views;
    sdfo::DeviceBuffer<int64_t> offs;
    // per-grid tile offsets for 128, 256 and 512 threads per CTA
    sdfo::DeviceBuffer<int64_t> tiles[3];
    int64_t ntiles[3] = {0, 0, 0};
};

namespace sdfo {
namespace {

int shape_index(int threads) { return threads == 128 ? 0 : (threads == 256 ? 1 : 2); }

template <int MODE, int THREADS>
__global__ void __launch_bounds__(THREADS)
    k_query_batch(const GridView* __restrict__ views, const int64_t* __restrict__ offs,
                  const int64_t* __restrict__ tiles, int n, const sdfo_pose* __restrict__ poses,
                  const float* __restrict__ pts, float* __restrict__ gap, float* __restrict__ grad,
                  uint8_t* __restrict__ valid)
{
    __shared__ GridView sv;
    __shared__ double sR[9], st[3];
    const int g = find_segment(tiles, n, blockIdx.x);
    if (threadIdx.x == 0)
    {
        sv = views[g];
        for (int a = 0; a < 9; ++a) sR[a] = poses ? poses[g].R[a] : ((a % 4) == 0 ? 1.0 : 0.0);
        for (int a = 0; a < 3; ++a) st[a] = poses ? poses[g].t[a] : 0.0;
    }
    __syncthreads();
    const int64_t q = offs[g] + (int64_t)(blockIdx.x - tiles[g]) * THREADS + threadIdx.x;
    if (q >= offs[g + 1]) return;
    const double w[3] = {(double)__ldcs(pts + 3 * q) - st[0], (double)__ldcs(pts + 3 * q + 1) - st[1],
                         (double)__ldcs(pts + 3 * q + 2) - st[2]};
    // p = R^T (x - t)
    const double p[3] = {sR[0] * w[0] + sR[3] * w[1] + sR[6] * w[2],
                         sR[1] * w[0] + sR[4] * w[1] + sR[7] * w[2],
                         sR[2] * w[0] + sR[5] * w[1] + sR[8] * w[2]};
    Interp r;
    float unit[3];
    bool ok;
    if (sv.layout == SDFO_LAYOUT_DENSE)
        ok = evaluate<MODE, false, 0, false>(sv, p, r, unit);
    else if (sv.bd == 8)
        ok = evaluate<MODE, true, 8, false>(sv, p, r, unit);
    else
        ok = evaluate<MODE, true, 0, false>(sv, p, r, unit);
    if (!ok)
    {
        r.gap = 0.f;
        r.g[0] = r.g[1] = r.g[2] = 0.f;
    }
    __stcs(gap + q, r.gap);
    if (grad)
    {
        // world gradient R g
        __stcs(grad + 3 * q + 0, (float)(sR[0] * r.g[0] + sR[1] * r.g[1] + sR[2] * r.g[2]));
        __stcs(grad + 3 * q + 1, (float)(sR[3] * r.g[0] + sR[4] * r.g[1] + sR[5] * r.g[2]));
        __stcs(grad + 3 * q + 2, (float)(sR[6] * r.g[0] + sR[7] * r.g[1] + sR[8] * r.g[2]));
    }
    if (valid) valid[q] = ok ? 1 : 0;
}

template <int MODE>
void launch_batch(const sdfo_query_batch* b, const float* pts, const sdfo_pose* poses, float* gap,
                  float* grad, uint8_t* valid, cudaStream_t s)
{
    const int si = shape_index(b->threads);
    const unsigned blocks = (unsigned)b->ntiles[si];
    if (blocks == 0) return;
    const GridView* v = b->views.get();
    const int64_t* o = b->offs.get();
    const int64_t* t = b->tiles[si].get();
    switch (b->threads)
    {
    case 128:
        k_query_batch<MODE, 128><<<blocks, 128, 0, s>>>(v, o, t, b->n, poses, pts, gap, grad, valid);
        break;
    case 512:
        k_query_batch<MODE, 512><<<blocks, 512, 0, s>>>(v, o, t, b->n, poses, pts, gap, grad, valid);
        break;
    default:
        k_query_batch<MODE, 256><<<blocks, 256, 0, s>>>(v, o, t, b->n, poses, pts, gap, grad, valid);
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
        std::vector<int64_t> offs((size_t)n + 1, 0);
        std::vector<int64_t> tiles[3];
        const int shapes[3] = {128, 256, 512};
        for (int k = 0; k < 3; ++k) tiles[k].assign((size_t)n + 1, 0);
        for (int g = 0; g < n; ++g)
        {
            SDFO_REQUIRE(grids[g] != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
            SDFO_REQUIRE(h_counts[g] >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
            SDFO_REQUIRE(g == 0 || grids[g]->device == grids[0]->device, SDFO_ERR_INVALID_ARGUMENT,
                         "grids of a query batch must be on one device");
            views[(size_t)g] = make_view(grids[g]);
            offs[(size_t)g + 1] = offs[(size_t)g] + h_counts[g];
            for (int k = 0; k < 3; ++k)
                tiles[k][(size_t)g + 1] = tiles[k][(size_t)g] + (h_counts[g] + shapes[k] - 1) / shapes[k];
        }
        b->device = grids[0]->device;
        b->total = offs[(size_t)n];
        SDFO_REQUIRE(tiles[0][(size_t)n] < (int64_t(1) << 31), SDFO_ERR_INVALID_ARGUMENT,
                     "too many queries in one batch");
        b->views.reset((size_t)n);
        b->offs.reset((size_t)n + 1);
        SDFO_CUDA(cudaMemcpy(b->views.get(), views.data(), sizeof(GridView) * n, cudaMemcpyHostToDevice));
        SDFO_CUDA(cudaMemcpy(b->offs.get(), offs.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
        for (int k = 0; k < 3; ++k)
        {
            b->tiles[k].reset((size_t)n + 1);
            b->ntiles[k] = tiles[k][(size_t)n];
            SDFO_CUDA(cudaMemcpy(b->tiles[k].get(), tiles[k].data(), sizeof(int64_t) * (n + 1),
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
