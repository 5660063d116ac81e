// The saved-linearisation backward for points (dL/dp = dgap * grad +
// H dgrad) as a bulk-copy pipeline: persistent CTAs stream tiles of 256
// queries through shared memory with cp.async.bulk (TMA bulk copies, no
// tensor map, no multicast) completing on mbarriers, three tiles in flight per
// CTA, and write the results back with bulk stores.  The per-query work is
// 15 FMAs against 64 bytes of traffic, so the kernel's only job is to keep
// enough bytes in flight to run at copy bandwidth.  The last n mod 256
// queries take plain loads and stores in one extra CTA of the same launch.
//
// Every wait on an mbarrier is bounded: a wait that runs out sets bit 0 of
// the device status word (sdfo_device_status), waits (bounded) for the CTA's
// outstanding bulk stores and returns.
#include "bulk.cuh"
#include "sdfo_internal.cuh"

namespace sdfo {

__device__ unsigned int g_device_status = 0;

namespace {

using namespace bulk;

constexpr int kTile = 256;   // queries per tile (= threads per CTA)
constexpr int kStages = 3;
constexpr unsigned kWaitLimit = 1u << 24;
// Test-only: {main-loop wait limit (0 = kWaitLimit), withhold the first
// tile's loads in every CTA}; both 0 in normal operation.
__device__ unsigned int g_bwd_test[2] = {0u, 0u};

// Shared-memory layout of one input stage (bytes): dgap | dgrad | grad | hess6.
constexpr int kOffDgap = 0;
constexpr int kOffDgrad = kOffDgap + 4 * kTile;
constexpr int kOffGrad = kOffDgrad + 12 * kTile;
constexpr int kOffHess = kOffGrad + 12 * kTile;
constexpr int kStageBytes = kOffHess + 24 * kTile; // 13 KB
constexpr int kOutBytes = 12 * kTile;              // 3 KB, double-buffered

// One tile's loads into stage `s`: dgap (if any), dgrad (if any), grad, hess6.
__device__ __forceinline__ void issue_tile(unsigned char* stage, uint64_t* bar, int64_t q0, const float* dgap,
                                           const float* dgrad, const float* grad, const float* hess6)
{
    const unsigned bytes = (dgap ? 4u : 0u) * kTile + (dgrad ? 12u : 0u) * kTile + 36u * kTile;
    mbar_expect_tx(bar, bytes);
    if (dgap) bulk_load(stage + kOffDgap, dgap + q0, 4 * kTile, bar);
    if (dgrad) bulk_load(stage + kOffDgrad, dgrad + 3 * q0, 12 * kTile, bar);
    bulk_load(stage + kOffGrad, grad + 3 * q0, 12 * kTile, bar);
    bulk_load(stage + kOffHess, hess6 + 6 * q0, 24 * kTile, bar);
}

__global__ void __launch_bounds__(kTile) k_backward_saved_bulk(int64_t n, const float* __restrict__ grad,
                                                               const float* __restrict__ hess6,
                                                               const float* __restrict__ dgap,
                                                               const float* __restrict__ dgrad,
                                                               float* __restrict__ dpts)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[kStages];
    __shared__ int s_abort;
    __shared__ long long s_kabort; // the tile whose wait ran out
    __shared__ unsigned s_limit;
    __shared__ int s_withhold;
    unsigned char* stages = smem;
    unsigned char* outs = smem + kStages * kStageBytes;
    const int64_t tiles = n / kTile;
    const bool rem = (n % kTile) != 0;
    if (rem && blockIdx.x == gridDim.x - 1)
    {
        // the remainder, one query per thread
        const int64_t q = tiles * kTile + threadIdx.x;
        if (q >= n) return;
        const float dG = dgap ? dgap[q] : 0.f;
        float dg[3] = {0.f, 0.f, 0.f};
        if (dgrad)
            for (int a = 0; a < 3; ++a) dg[a] = dgrad[3 * q + a];
        const float* gr = grad + 3 * q;
        const float* H = hess6 + 6 * q;
        dpts[3 * q] = dG * gr[0] + H[0] * dg[0] + H[1] * dg[1] + H[2] * dg[2];
        dpts[3 * q + 1] = dG * gr[1] + H[1] * dg[0] + H[3] * dg[1] + H[4] * dg[2];
        dpts[3 * q + 2] = dG * gr[2] + H[2] * dg[0] + H[4] * dg[1] + H[5] * dg[2];
        return;
    }
    const int64_t first = blockIdx.x, step = gridDim.x - (rem ? 1 : 0);
    const int64_t mine = first < tiles ? (tiles - first + step - 1) / step : 0;
    if (threadIdx.x == 0)
    {
        s_abort = 0;
        s_limit = g_bwd_test[0] ? g_bwd_test[0] : kWaitLimit;
        s_withhold = g_bwd_test[1] != 0u;
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int k = s_withhold ? 1 : 0; k < kStages && k < mine; ++k)
            issue_tile(stages + k * kStageBytes, &bars[k], (first + k * step) * kTile, dgap, dgrad, grad, hess6);
    }
    __syncthreads();
    for (int64_t k = 0; k < mine; ++k)
    {
        const int s = (int)(k % kStages);
        const unsigned parity = (unsigned)((k / kStages) & 1);
        unsigned it = 0;
        while (!mbar_try_wait(&bars[s], parity))
            if (++it >= s_limit)
            {
                s_abort = 1; // benign race: every writer stores the same values
                s_kabort = k;
                break;
            }
        __syncthreads();
        if (s_abort) break;
        const unsigned char* st = stages + s * kStageBytes;
        const int t = threadIdx.x;
        const float dG = dgap ? reinterpret_cast<const float*>(st + kOffDgap)[t] : 0.f;
        float dg[3] = {0.f, 0.f, 0.f};
        if (dgrad)
            for (int a = 0; a < 3; ++a) dg[a] = reinterpret_cast<const float*>(st + kOffDgrad)[3 * t + a];
        const float* gr = reinterpret_cast<const float*>(st + kOffGrad) + 3 * t;
        const float* H = reinterpret_cast<const float*>(st + kOffHess) + 6 * t;
        const float o0 = dG * gr[0] + H[0] * dg[0] + H[1] * dg[1] + H[2] * dg[2];
        const float o1 = dG * gr[1] + H[1] * dg[0] + H[3] * dg[1] + H[4] * dg[2];
        const float o2 = dG * gr[2] + H[2] * dg[0] + H[4] * dg[1] + H[5] * dg[2];
        const int ob = (int)(k & 1);
        float* out = reinterpret_cast<float*>(outs + ob * kOutBytes);
        if (threadIdx.x == 0 && k >= 2) bulk_wait_read<1>(); // the store that used this buffer is done
        __syncthreads();
        out[3 * t] = o0;
        out[3 * t + 1] = o1;
        out[3 * t + 2] = o2;
        fence_async_shared();
        __syncthreads(); // stage s consumed, output written
        if (threadIdx.x == 0)
        {
            const int64_t q0 = (first + k * step) * kTile;
            bulk_store(dpts + 3 * q0, out, kOutBytes);
            bulk_commit();
            const int64_t nk = k + kStages;
            if (nk < mine)
                issue_tile(stages + s * kStageBytes, &bars[s], (first + nk * step) * kTile, dgap, dgrad, grad,
                           hess6);
        }
    }
    if (threadIdx.x == 0)
    {
        if (s_abort)
        {
            atomicOr(&g_device_status, 1u);
            // the tiles issued but not consumed (s_kabort .. s_kabort + kStages
            // - 1) complete into this CTA's shared memory: wait for them
            // (bounded) before the CTA exits
            for (long long j = s_kabort; j < s_kabort + kStages && j < mine; ++j)
            {
                if (j == 0 && s_withhold) continue; // nothing in flight
                unsigned it = 0;
                while (!mbar_try_wait(&bars[j % kStages], (unsigned)((j / kStages) & 1)) && ++it < kWaitLimit)
                {
                }
            }
        }
        bulk_wait_read<0>();
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
}

} // namespace

bool launch_backward_saved_bulk(int64_t n, const float* grad, const float* hess6, const float* dgap,
                                const float* dgrad, float* dpts, cudaStream_t s)
{
    auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    if (n < kTile || !grad || !hess6 || !dpts || !a16(grad) || !a16(hess6) || !a16(dpts) ||
        (dgap && !a16(dgap)) || (dgrad && !a16(dgrad)))
        return false;
    const int64_t tiles = n / kTile;
    const int sms = current_sm_count();
    const int smem = kStages * kStageBytes + 2 * kOutBytes; // 45 KB
    const int64_t rem = n % kTile ? 1 : 0; // one more CTA, for the remainder
    const int64_t ctas = std::min<int64_t>(tiles, (int64_t)sms * 4 - rem) + rem;
    k_backward_saved_bulk<<<(unsigned)ctas, kTile, smem, s>>>(n, grad, hess6, dgap, dgrad, dpts);
    SDFO_CHECK_LAUNCH();
    return true;
}

void set_backward_bulk_wait_test(unsigned limit, int withhold_first_tile)
{
    const unsigned v[2] = {limit, withhold_first_tile ? 1u : 0u};
    SDFO_CUDA(cudaMemcpyToSymbol(g_bwd_test, v, sizeof(v)));
}

} // namespace sdfo

extern "C" int sdfo_debug_wait_test(uint32_t wait_limit, int32_t withhold_first_tile)
{
    return sdfo::guarded([&] {
        sdfo::set_query_pipe_wait_test(wait_limit, withhold_first_tile);
        sdfo::set_backward_bulk_wait_test(wait_limit, withhold_first_tile);
    });
}

extern "C" int sdfo_device_status(uint32_t* flags, int32_t clear)
{
    return sdfo::guarded([&] {
        SDFO_REQUIRE(flags != nullptr, SDFO_ERR_INVALID_ARGUMENT, "flags is NULL");
        unsigned v = 0;
        SDFO_CUDA(cudaMemcpyFromSymbol(&v, sdfo::g_device_status, sizeof(v)));
        *flags = v | sdfo::query_pipe_status(clear != 0);
        if (clear)
        {
            const unsigned z = 0;
            SDFO_CUDA(cudaMemcpyToSymbol(sdfo::g_device_status, &z, sizeof(z)));
        }
    });
}
