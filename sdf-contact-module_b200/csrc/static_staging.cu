// sdfo_query_host_static: the host-buffer query without any device
// allocation.
//
// sdfo_query_host stages the caller's host points and results through device
// memory that the library allocates (once per grid handle, with cudaMalloc).
// Some callers cannot let a library allocate device memory: applications that
// hand all of the GPU's memory to their own pool at start-up, hosts that
// forbid allocations (and the synchronisation cudaMalloc implies) inside their
// time-step loop, or plugins whose allocation budget is fixed by the host.
// This variant stages through one file-scope device array of fixed size
// instead, so it performs no cudaMalloc / cudaFree and no allocating library
// call.  The array is part of the module image: every GPU that loads
// libsdfo_cuda holds its kStaticStagingBytes until the process exits.
#include <cstring>
#include <mutex>

#include "sdfo_internal.cuh"

namespace sdfo {
namespace {

constexpr size_t kStaticStagingBytes = size_t(SDFO_STATIC_STAGING_BYTES);

// Shared by every call on a device; it keeps the last call's contents.
static __device__ __align__(256) unsigned char g_static_staging[kStaticStagingBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_staging_addr[kMaxDevices] = {};

// Device address of the array for the current device.  In host code
// g_static_staging names a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
void* staging_address()
{
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    SDFO_REQUIRE(dev >= 0 && dev < kMaxDevices, SDFO_ERR_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_staging_addr[dev] == nullptr)
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_staging);
        if (e != cudaSuccess)
        {
            (void)cudaGetLastError();
            throw Error(SDFO_ERR_CUDA, std::string("cudaGetSymbolAddress of the static staging "
                                                   "array failed: ") + cudaGetErrorString(e));
        }
        g_staging_addr[dev] = p;
    }
    return g_staging_addr[dev];
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

} // namespace
} // namespace sdfo

using namespace sdfo;

extern "C" int sdfo_query_host_static(const sdfo_grid* g, int32_t mode, const void* h_points,
                                      int32_t points_f64, int64_t n, float* h_gap, float* h_grad,
                                      uint8_t* h_valid, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(g != nullptr, SDFO_ERR_INVALID_ARGUMENT, "grid is NULL");
        SDFO_REQUIRE(n >= 0, SDFO_ERR_INVALID_ARGUMENT, "negative query count");
        if (n == 0) return;
        SDFO_REQUIRE(h_points && h_gap, SDFO_ERR_INVALID_ARGUMENT, "points and gap are required");
        SDFO_REQUIRE(mode >= SDFO_FIRST_ORDER && mode <= SDFO_CONTACT_AWARE,
                     SDFO_ERR_INVALID_ARGUMENT, "unknown query mode");
        int dev = 0;
        SDFO_CUDA(cudaGetDevice(&dev));
        SDFO_REQUIRE(dev == g->device, SDFO_ERR_INVALID_ARGUMENT,
                     "the grid's device must be the current device");
        const size_t pb = (size_t)n * 3 * (points_f64 ? sizeof(double) : sizeof(float));
        const size_t gb = sizeof(float) * (size_t)n, vb = 3 * gb;
        const size_t need = up256(pb) + up256(gb) + (h_grad ? up256(vb) : 0) +
                            (h_valid ? up256((size_t)n) : 0);
        if (need > kStaticStagingBytes)
            throw Error(SDFO_ERR_INVALID_ARGUMENT,
                        "sdfo_query_host_static: " + std::to_string(n) +
                            " queries need " + std::to_string(need) +
                            " bytes of staging, above the static limit of " +
                            std::to_string(kStaticStagingBytes) +
                            " bytes; split the batch or use sdfo_query_host");
        unsigned char* base = static_cast<unsigned char*>(staging_address());
        auto take = [&](size_t b) {
            unsigned char* p = base;
            base += up256(b);
            return p;
        };
        void* pts = take(pb);
        float* gap = reinterpret_cast<float*>(take(gb));
        float* grad = h_grad ? reinterpret_cast<float*>(take(vb)) : nullptr;
        uint8_t* valid = h_valid ? take((size_t)n) : nullptr;
        // A launch that completes writes every output element, so nothing in
        // the array has to start at zero.  A pipelined launch whose bounded
        // wait ran out stops early and leaves earlier calls' contents in
        // part of the outputs: the status word, read below in stream order,
        // turns that into SDFO_ERR_DEVICE_STATUS instead of results.
        cudaStream_t s = as_stream(stream);
        unsigned* status_dev = query_pipe_status_address();
        SDFO_CUDA(cudaMemcpyAsync(pts, h_points, pb, cudaMemcpyHostToDevice, s));
        const QueryOutputs o{gap, grad, nullptr, nullptr, valid, nullptr};
        launch_query(make_view(g), mode, pts, points_f64 != 0, n, o, s);
        SDFO_CUDA(cudaMemcpyAsync(h_gap, gap, gb, cudaMemcpyDeviceToHost, s));
        if (h_grad) SDFO_CUDA(cudaMemcpyAsync(h_grad, grad, vb, cudaMemcpyDeviceToHost, s));
        if (h_valid) SDFO_CUDA(cudaMemcpyAsync(h_valid, valid, (size_t)n, cudaMemcpyDeviceToHost, s));
        unsigned status = 0;
        SDFO_CUDA(cudaMemcpyAsync(&status, status_dev, sizeof(status), cudaMemcpyDeviceToHost, s));
        SDFO_CUDA(cudaStreamSynchronize(s));
        if (status & kPipeStatusWaitAbort)
        {
            SDFO_CUDA(cudaMemsetAsync(status_dev, 0, sizeof(unsigned), s));
            SDFO_CUDA(cudaStreamSynchronize(s));
            throw Error(SDFO_ERR_DEVICE_STATUS,
                        "a bounded wait of the pipelined query kernel ran out; the results are incomplete");
        }
    });
}
