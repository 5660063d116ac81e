// sdfo_query_host: the query with host buffers (SdfOracle::queryBatch over
// caller-owned host arrays, SdfOracle.cpp:434-444), and the process-wide
// tuning knobs (sdfo_set_tuning).
//
// With pinned host buffers and more points than one chunk, the call is a
// three-stream pipeline over chunks: the caller's stream copies the chunks'
// points in back to back, the handle's query stream runs each chunk's query
// once its points have arrived, and the handle's copy-out stream copies each
// chunk's results back once its query is done (events between the streams).
// Host-to-device and device-to-host copies then run at the same time on
// separate copy engines, so a step costs about the larger of the two
// transfers instead of their sum.  The first chunk has
// `host_chunk_queries` points and each next one `host_chunk_growth_pct`
// percent of the previous: a small first chunk starts the copy-out early,
// larger later ones keep the number of copies (each with a fixed cost) low,
// and the copy-out (the larger transfer: 17 bytes per query against 12) is
// never left waiting.  Pageable buffers (whose copies the driver stages
// synchronously) and batches of one chunk take one copy in, one launch and
// one copy out on the caller's stream.
//
// Pinned host memory is mapped into the device on 64-bit systems, so the
// query can also use the caller's buffers in place (sdfo_tuning.host_io_mode):
// mode 2 writes each chunk's results straight to the host (no copy-out
// stream); mode 3 is one launch that reads the points from the host and
// writes the results back while it runs, which keeps both directions of the
// bus busy without staging, chunking or per-copy setup.  Those launches use
// the plain query kernel (ordinary stores), never bulk-copy transfers.
//
// The call is synchronous.  Before it returns it reads the pipelined query
// kernel's status word in stream order; a bounded wait that ran out in a
// launch since the word was last cleared is reported as
// SDFO_ERR_DEVICE_STATUS (the word is then cleared), so stale staging
// contents are never returned as results.
#include <algorithm>
#include <atomic>
#include <string>

#include "sdfo_internal.cuh"

namespace sdfo {

namespace {

constexpr int kMaxChunks = 64;
constexpr int64_t kDefaultHostChunk = 32768;
constexpr int kDefaultChunkGrowth = 130; // percent
std::atomic<int64_t> g_host_chunk{kDefaultHostChunk};
std::atomic<int> g_chunk_growth{kDefaultChunkGrowth};

int64_t round_up256(int64_t v) { return (v + 255) & ~int64_t(255); }

// host io mode - 1: 0 copies, 1 results written in place, 2 both ways in place
// default 3 (zero-copy): 2.26 G queries/s for the 1M-point hollow-cylinder
// batch, against 2.23 (results written in place) and 2.02 (staged copies)
constexpr int kDefaultIoMode = 2;
std::atomic<int> g_output_mode{kDefaultIoMode};

// Device address of pinned host memory mapped into the device (NULL for
// pageable memory or when it is not mapped); `pinned` receives whether the
// memory is page-locked host memory.
void* mapped_address(const void* p, bool& pinned)
{
    pinned = false;
    if (p == nullptr) return nullptr;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        (void)cudaGetLastError();
        return nullptr;
    }
    pinned = a.type == cudaMemoryTypeHost;
    return pinned ? a.devicePointer : nullptr;
}

} // namespace

struct HostPipe
{
    cudaStream_t comp = nullptr; // the chunks' queries
    cudaStream_t out = nullptr;  // device-to-host copies of finished chunks
    cudaEvent_t start = nullptr; // the caller's stream reached the call
    cudaEvent_t in[kMaxChunks] = {};    // chunk's points copied in
    cudaEvent_t ready[kMaxChunks] = {}; // chunk's results written
    unsigned* status = nullptr; // pinned host copy of the query status word
};

void destroy_host_pipe(HostPipe* p)
{
    if (!p) return;
    for (cudaEvent_t& e : p->ready)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t& e : p->in)
        if (e) cudaEventDestroy(e);
    if (p->start) cudaEventDestroy(p->start);
    if (p->comp) cudaStreamDestroy(p->comp);
    if (p->out) cudaStreamDestroy(p->out);
    if (p->status) cudaFreeHost(p->status);
    delete p;
}

namespace {

// The handle's pipe (created on its first host query; the caller holds
// ws_mutex).
HostPipe* host_pipe(const sdfo_grid* g)
{
    if (g->host_pipe) return g->host_pipe;
    auto* p = new HostPipe();
    try
    {
        SDFO_CUDA(cudaStreamCreateWithFlags(&p->comp, cudaStreamNonBlocking));
        SDFO_CUDA(cudaStreamCreateWithFlags(&p->out, cudaStreamNonBlocking));
        SDFO_CUDA(cudaEventCreateWithFlags(&p->start, cudaEventDisableTiming));
        for (cudaEvent_t& e : p->ready) SDFO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (cudaEvent_t& e : p->in) SDFO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        SDFO_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&p->status), sizeof(unsigned), cudaHostAllocDefault));
        *p->status = 0;
    }
    catch (...)
    {
        destroy_host_pipe(p);
        throw;
    }
    g->host_pipe = p;
    return p;
}

struct Staging
{
    unsigned char* pts;
    float* gap;
    float* grad;
    float* unit;
    float* wit;
    uint8_t* valid;
};

} // namespace

} // namespace sdfo

using namespace sdfo;

extern "C" {

int sdfo_query_host(const sdfo_grid* g, int32_t mode, const void* h_points, int32_t points_f64,
                    int64_t n, float* h_gap, float* h_grad, float* h_unit, float* h_witness,
                    uint8_t* h_valid, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(g != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
        SDFO_REQUIRE(g->stored_voxels > 0 || g->info.layout == SDFO_LAYOUT_SPARSE,
                     SDFO_ERR_INVALID_ARGUMENT, "grid is empty");
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(h_points && h_gap, SDFO_ERR_INVALID_ARGUMENT, "points and gap are required");
        SDFO_REQUIRE(mode >= SDFO_FIRST_ORDER && mode <= SDFO_CONTACT_AWARE,
                     SDFO_ERR_INVALID_ARGUMENT, "unknown query mode");
        SDFO_REQUIRE(n <= (int64_t)65535 * 256 * 4096, SDFO_ERR_INVALID_ARGUMENT, "too many queries");
        cudaStream_t s = as_stream(stream);
        const size_t ep = points_f64 ? sizeof(double) : sizeof(float);
        // pinned buffers take the pipeline; sdfo_tuning.host_io_mode 2 and 3
        // (every output mapped into the device) let the query write the
        // results straight into them, 3 also read the points in place
        bool pinned = true;
        void* mapped[5] = {};
        {
            float* outs[5] = {h_gap, h_grad, h_unit, h_witness, reinterpret_cast<float*>(h_valid)};
            bool pp = false;
            (void)mapped_address(h_points, pp);
            pinned = pp;
            for (int k = 0; k < 5; ++k)
                if (outs[k])
                {
                    mapped[k] = mapped_address(outs[k], pp);
                    pinned = pinned && pp;
                }
        }
        const bool outs_mapped = mapped[0] && (!h_grad || mapped[1]) && (!h_unit || mapped[2]) &&
                                 (!h_witness || mapped[3]) && (!h_valid || mapped[4]);
        bool pp = false;
        void* pts_mapped = mapped_address(h_points, pp);
        const int io = g_output_mode.load();
        // io 2: the pipeline's queries write the results into the caller's
        // buffers; io 3: one query launch reads the points from and writes
        // the results to the caller's buffers, over the bus both ways at once
        const bool direct = pinned && io >= 1 && outs_mapped;
        const bool zero_copy = direct && io == 2 && pts_mapped != nullptr;
        // one staging allocation per handle, 256-byte aligned sub-buffers
        auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t pb = (size_t)n * 3 * ep;
        const size_t gb = sizeof(float) * (size_t)n, vb = sizeof(float) * 3 * (size_t)n;
        const size_t need = zero_copy ? 0
                            : direct ? up(pb)
                                     : up(pb) + up(gb) + (h_grad ? up(vb) : 0) + (h_unit ? up(vb) : 0) +
                                           (h_witness ? up(vb) : 0) + (h_valid ? up((size_t)n) : 0);
        std::lock_guard<std::mutex> lock(g->ws_mutex);
        HostPipe* hp = host_pipe(g);
        if (g->ws_bytes < need)
        {
            SDFO_CUDA(cudaStreamSynchronize(s));
            device_free(g->ws);
            g->ws = nullptr;
            g->ws_bytes = 0;
            g->ws = device_alloc(need);
            g->ws_bytes = need;
        }
        unsigned char* base = static_cast<unsigned char*>(g->ws);
        auto take = [&](size_t b) {
            unsigned char* p = base;
            base += up(b);
            return p;
        };
        Staging d{};
        d.pts = zero_copy ? static_cast<unsigned char*>(pts_mapped) : take(pb);
        if (direct)
        {
            d.gap = static_cast<float*>(mapped[0]);
            d.grad = static_cast<float*>(mapped[1]);
            d.unit = static_cast<float*>(mapped[2]);
            d.wit = static_cast<float*>(mapped[3]);
            d.valid = static_cast<uint8_t*>(mapped[4]);
        }
        else
        {
            d.gap = reinterpret_cast<float*>(take(gb));
            d.grad = h_grad ? reinterpret_cast<float*>(take(vb)) : nullptr;
            d.unit = h_unit ? reinterpret_cast<float*>(take(vb)) : nullptr;
            d.wit = h_witness ? reinterpret_cast<float*>(take(vb)) : nullptr;
            d.valid = h_valid ? take((size_t)n) : nullptr;
        }
        const GridView view = make_view(g);
        unsigned* status_dev = query_pipe_status_address();

        int64_t chunk = round_up256(std::max<int64_t>(256, g_host_chunk.load()));
        // outputs of `m` queries starting at q0, to host on stream `t`
        auto copy_out = [&](int64_t q0, int64_t m, cudaStream_t t) {
            const size_t f = sizeof(float);
            SDFO_CUDA(cudaMemcpyAsync(h_gap + q0, d.gap + q0, f * m, cudaMemcpyDeviceToHost, t));
            if (h_grad)
                SDFO_CUDA(cudaMemcpyAsync(h_grad + 3 * q0, d.grad + 3 * q0, 3 * f * m, cudaMemcpyDeviceToHost, t));
            if (h_unit)
                SDFO_CUDA(cudaMemcpyAsync(h_unit + 3 * q0, d.unit + 3 * q0, 3 * f * m, cudaMemcpyDeviceToHost, t));
            if (h_witness)
                SDFO_CUDA(cudaMemcpyAsync(h_witness + 3 * q0, d.wit + 3 * q0, 3 * f * m, cudaMemcpyDeviceToHost,
                                          t));
            if (h_valid) SDFO_CUDA(cudaMemcpyAsync(h_valid + q0, d.valid + q0, (size_t)m, cudaMemcpyDeviceToHost, t));
        };
        auto query = [&](int64_t q0, int64_t m, cudaStream_t t) {
            const QueryOutputs o{d.gap + q0,
                                 d.grad ? d.grad + 3 * q0 : nullptr,
                                 d.unit ? d.unit + 3 * q0 : nullptr,
                                 d.wit ? d.wit + 3 * q0 : nullptr,
                                 d.valid ? d.valid + q0 : nullptr,
                                 nullptr, nullptr, direct};
            launch_query(view, mode, d.pts + (size_t)q0 * 3 * ep, points_f64 != 0, m, o, t);
        };
        cudaStream_t last = s;
        if (zero_copy)
        {
            query(0, n, s);
        }
        else if (!pinned || n <= chunk)
        {
            SDFO_CUDA(cudaMemcpyAsync(d.pts, h_points, pb, cudaMemcpyHostToDevice, s));
            query(0, n, s);
            if (!direct) copy_out(0, n, s);
        }
        else
        {
            // chunk boundaries: growing by g percent from `chunk`, multiples
            // of 256 (whole tiles of the pipelined kernel), the last chunk
            // taking the rest once kMaxChunks - 1 are placed
            const int g = std::max(100, g_chunk_growth.load());
            int64_t bounds[kMaxChunks + 1];
            int nc = 0;
            bounds[0] = 0;
            for (double size = (double)chunk; bounds[nc] < n;)
            {
                int64_t m = nc + 1 == kMaxChunks ? n - bounds[nc] : round_up256((int64_t)size);
                m = std::min(m, n - bounds[nc]);
                bounds[nc + 1] = bounds[nc] + m;
                ++nc;
                size = size * g / 100.0;
            }
            const unsigned char* hp_pts = static_cast<const unsigned char*>(h_points);
            SDFO_CUDA(cudaEventRecord(hp->start, s));
            SDFO_CUDA(cudaStreamWaitEvent(hp->comp, hp->start, 0));
            SDFO_CUDA(cudaStreamWaitEvent(hp->out, hp->start, 0));
            for (int c = 0; c < nc; ++c)
            {
                const int64_t q0 = bounds[c], m = bounds[c + 1] - q0;
                SDFO_CUDA(cudaMemcpyAsync(d.pts + (size_t)q0 * 3 * ep, hp_pts + (size_t)q0 * 3 * ep,
                                          (size_t)m * 3 * ep, cudaMemcpyHostToDevice, s));
                SDFO_CUDA(cudaEventRecord(hp->in[c], s));
                SDFO_CUDA(cudaStreamWaitEvent(hp->comp, hp->in[c], 0));
                query(q0, m, hp->comp);
                if (direct) continue; // the query wrote the results to the host
                SDFO_CUDA(cudaEventRecord(hp->ready[c], hp->comp));
                SDFO_CUDA(cudaStreamWaitEvent(hp->out, hp->ready[c], 0));
                copy_out(q0, m, hp->out);
            }
            last = direct ? hp->comp : hp->out;
        }
        // the status word after the last launch, in stream order
        SDFO_CUDA(cudaMemcpyAsync(hp->status, status_dev, sizeof(unsigned), cudaMemcpyDeviceToHost, last));
        SDFO_CUDA(cudaStreamSynchronize(last));
        if (*hp->status & kPipeStatusWaitAbort)
        {
            SDFO_CUDA(cudaMemsetAsync(status_dev, 0, sizeof(unsigned), s));
            SDFO_CUDA(cudaStreamSynchronize(s));
            throw Error(SDFO_ERR_DEVICE_STATUS,
                        "a bounded wait of the pipelined query kernel ran out; the results are incomplete");
        }
    });
}

int sdfo_set_tuning(const sdfo_tuning* t)
{
    return guarded([&] {
        // every field is checked before any is applied
        SDFO_REQUIRE(t != nullptr, SDFO_ERR_INVALID_ARGUMENT, "tuning is NULL");
        SDFO_REQUIRE(t->host_chunk_queries >= 0, SDFO_ERR_INVALID_ARGUMENT,
                     "host_chunk_queries must be >= 0");
        SDFO_REQUIRE(t->fill_ctas_per_sm >= 0 && t->fill_ctas_per_sm <= 64, SDFO_ERR_INVALID_ARGUMENT,
                     "CTAs per SM out of range");
        SDFO_REQUIRE(t->fill_tile_log2_x >= 0 && t->fill_tile_log2_y >= 0 &&
                         (t->fill_tile_log2_x > 0 ? t->fill_tile_log2_x : 3) +
                                 (t->fill_tile_log2_y > 0 ? t->fill_tile_log2_y : 3) <=
                             8,
                     SDFO_ERR_INVALID_ARGUMENT, "fill tile must hold at most 256 voxels in x and y");
        SDFO_REQUIRE(t->host_chunk_growth_pct == 0 || (t->host_chunk_growth_pct >= 100 && t->host_chunk_growth_pct <= 400),
                     SDFO_ERR_INVALID_ARGUMENT, "host_chunk_growth_pct must be 0 or in [100, 400]");
        SDFO_REQUIRE(t->host_io_mode >= 0 && t->host_io_mode <= 3, SDFO_ERR_INVALID_ARGUMENT,
                     "unknown host io mode");
        SDFO_REQUIRE(t->triangle_cull >= 0 && t->triangle_cull <= 2, SDFO_ERR_INVALID_ARGUMENT,
                     "triangle_cull must be 0, 1 or 2");
        SDFO_REQUIRE(t->sparse_pair_records >= 0 && t->sparse_pair_records <= 2, SDFO_ERR_INVALID_ARGUMENT,
                     "sparse_pair_records must be 0, 1 or 2");
        SDFO_REQUIRE(t->lbvh_traversal >= 0 && t->lbvh_traversal <= 2, SDFO_ERR_INVALID_ARGUMENT,
                     "unknown LBVH traversal");
        SDFO_REQUIRE(t->query_walk >= 0 && t->query_walk <= 2, SDFO_ERR_INVALID_ARGUMENT,
                     "query_walk must be 0, 1 or 2");
        g_host_chunk.store(t->host_chunk_queries > 0 ? t->host_chunk_queries : kDefaultHostChunk);
        g_chunk_growth.store(t->host_chunk_growth_pct > 0 ? t->host_chunk_growth_pct : kDefaultChunkGrowth);
        g_output_mode.store(t->host_io_mode == 0 ? kDefaultIoMode : t->host_io_mode - 1);
        set_triangle_cull(t->triangle_cull != 2);
        set_sparse_pair_records(t->sparse_pair_records);
        set_fill_ctas_per_sm(t->fill_ctas_per_sm);
        set_fill_tile(t->fill_tile_log2_x, t->fill_tile_log2_y);
        set_lbvh_stackless(t->lbvh_traversal != 1);
        set_query_walk(t->query_walk != 1);
    });
}

int sdfo_get_tuning(sdfo_tuning* t)
{
    return guarded([&] {
        SDFO_REQUIRE(t != nullptr, SDFO_ERR_INVALID_ARGUMENT, "tuning is NULL");
        *t = sdfo_tuning{};
        t->host_chunk_queries = (int32_t)g_host_chunk.load();
        t->host_chunk_growth_pct = g_chunk_growth.load();
        t->host_io_mode = g_output_mode.load() + 1;
        t->triangle_cull = triangle_cull() ? 1 : 2;
        t->sparse_pair_records = sparse_pair_records();
        t->fill_ctas_per_sm = fill_ctas_per_sm();
        int lx = 3, ly = 3;
        get_fill_tile(&lx, &ly);
        t->fill_tile_log2_x = lx;
        t->fill_tile_log2_y = ly;
        t->lbvh_traversal = lbvh_stackless() ? 2 : 1;
        t->query_walk = query_walk() ? 2 : 1;
    });
}

} // extern "C"
