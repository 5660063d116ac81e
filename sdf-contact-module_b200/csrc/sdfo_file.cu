// SDFO 0.1.0 files straight between disk and device grids: loadSdf /
// loadSparseSdf / SdfOracle::loadFromFile, saveSdf / saveSparseSdf and
// isValidSdf / isSparseSdf (SdfIO.cpp:93-552, SdfOracle.cpp:165-172) without
// the host SdfData / SparseSdfData detour.
//
// Load.  The 128-byte header is parsed and checked on the host in the
// reference's order and with its messages.  The payload is read with pread()
// by up to kMaxThreads threads, each owning two pinned staging slots and a
// stream, so that disk (page cache) reads, host-to-device copies and decoding
// overlap.  A dense file lands section by section in the grid's FP64 arrays
// (phi, normal, Hessian, witness and the contact-aware candidates), from which
// one kernel derives the FP32 {phi, n} query payload and FP32 Hessians.  A
// sparse file arrives in chunks of whole block records; a decoding kernel per
// chunk scatters them into the brick payload, Hessians and candidate arrays,
// and a last pair of kernels builds the block table (the first block with a
// given coordinate wins, as unordered_map::emplace in
// SparseSdfData::rebuildIndex, SdfData.h:172-183).  Candidate counts above the
// stride are found on the device and reported with the reference's messages;
// truncated files give the reference's header / payload errors.
//
// Save.  The reverse: sparse block records (and the dense u32 candidate
// counts) are packed on the device, copied into pinned slots and written with
// pwrite() at their file offsets, again by up to kMaxThreads threads.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <functional>
#include <thread>

#include "sdfo_internal.cuh"

namespace sdfo {
namespace {

// ---------------------------------------------------------------------------
// format constants (SdfIO.cpp:15-33, 60-91)
// ---------------------------------------------------------------------------
constexpr uint32_t kVersion = 100; // 0.1.0 as major*10000 + minor*100 + patch
constexpr uint32_t kFlagHessian = 1u << 0;
constexpr uint32_t kFlagSparse = 1u << 1;
constexpr uint32_t kFlagCandidates = 1u << 2;
constexpr uint32_t kLayoutDense = 1, kLayoutSparse = 2, kLayoutCaDense = 3, kLayoutCaSparse = 4;
constexpr int kMaxCandidates = 8; // SdfData::kMaxContactCandidates
constexpr int64_t kHeaderBytes = 128;
constexpr int64_t kBlockHeaderBytes = 16;

struct Header
{
    char magic[4];
    uint32_t version, nx, ny, nz, flags;
    double bmin[3], bmax[3], voxel[3];
    unsigned char reserved[32];
};

uint32_t get_u32(const unsigned char* b, int off)
{
    uint32_t v;
    std::memcpy(&v, b + off, 4);
    return v;
}

double get_f64(const unsigned char* b, int off)
{
    double v;
    std::memcpy(&v, b + off, 8);
    return v;
}

void put_u32(unsigned char* b, int off, uint32_t v) { std::memcpy(b + off, &v, 4); }
void put_f64(unsigned char* b, int off, double v) { std::memcpy(b + off, &v, 8); }

Header parse_header(const unsigned char* b)
{
    Header h;
    std::memcpy(h.magic, b, 4);
    h.version = get_u32(b, 4);
    h.nx = get_u32(b, 8);
    h.ny = get_u32(b, 12);
    h.nz = get_u32(b, 16);
    for (int a = 0; a < 3; ++a)
    {
        h.bmin[a] = get_f64(b, 20 + 8 * a);
        h.bmax[a] = get_f64(b, 44 + 8 * a);
        h.voxel[a] = get_f64(b, 68 + 8 * a);
    }
    h.flags = get_u32(b, 92);
    std::memcpy(h.reserved, b + 96, 32);
    return h;
}

void write_header(unsigned char* b, const sdfo_grid_info& info, uint32_t flags)
{
    std::memset(b, 0, kHeaderBytes);
    std::memcpy(b, "SDFO", 4);
    put_u32(b, 4, kVersion);
    for (int a = 0; a < 3; ++a) put_u32(b, 8 + 4 * a, (uint32_t)info.shape[a]);
    for (int a = 0; a < 3; ++a)
    {
        put_f64(b, 20 + 8 * a, info.bmin[a]);
        put_f64(b, 44 + 8 * a, info.bmax[a]);
        put_f64(b, 68 + 8 * a, info.voxel[a]);
    }
    put_u32(b, 92, flags);
}

[[noreturn]] void io_error(const std::string& msg) { throw Error(SDFO_ERR_IO, msg); }

// Milliseconds since the previous lap (load phases go to the grid's build
// statistics: setup = allocation, fill = file read + transfer, hessian =
// device decoding that follows the transfer).
struct Laps
{
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now(), t = t0;
    double lap()
    {
        const auto n = std::chrono::steady_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(n - t).count();
        t = n;
        return ms;
    }
    double total() const
    {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

// ---------------------------------------------------------------------------
// files
// ---------------------------------------------------------------------------
struct File
{
    int fd = -1;
    int64_t size = 0;
    unsigned char* map = nullptr; // writable mapping of an output file, or NULL
    File() = default;
    File(const File&) = delete;
    File& operator=(const File&) = delete;
    ~File()
    {
        if (map) ::munmap(map, (size_t)size);
        if (fd >= 0) ::close(fd);
    }
    // Unmaps and closes; false when closing reports an error.
    bool finish()
    {
        bool ok = true;
        if (map) ok = ::munmap(map, (size_t)size) == 0;
        map = nullptr;
        if (fd >= 0) ok = (::close(fd) == 0) && ok;
        fd = -1;
        return ok;
    }
};

// Reads up to n bytes at off; returns the number read (short only at EOF).
int64_t pread_full(int fd, void* dst, int64_t n, int64_t off)
{
    int64_t got = 0;
    while (got < n)
    {
        const ssize_t r = ::pread(fd, static_cast<char*>(dst) + got, (size_t)(n - got), (off_t)(off + got));
        if (r < 0)
        {
            if (errno == EINTR) continue;
            io_error(std::string("read error: ") + std::strerror(errno));
        }
        if (r == 0) break;
        got += r;
    }
    return got;
}

void pwrite_full(int fd, const void* src, int64_t n, int64_t off)
{
    int64_t put = 0;
    while (put < n)
    {
        const ssize_t r = ::pwrite(fd, static_cast<const char*>(src) + put, (size_t)(n - put), (off_t)(off + put));
        if (r < 0)
        {
            if (errno == EINTR) continue;
            io_error(std::string("Failed to write SdfOracle data file: ") + std::strerror(errno));
        }
        put += r;
    }
}

// ---------------------------------------------------------------------------
// pinned staging (process-wide; one file transfer at a time)
// ---------------------------------------------------------------------------
constexpr int kMaxThreads = 4;
constexpr int64_t kSlotBytes = 8ll << 20;

// Mapped pinned memory: dense sections are copied from / to it with
// cudaMemcpyAsync; sparse block records are decoded from it, and packed into
// it, by kernels reading and writing it over the bus (no device staging).
struct PinnedPool
{
    std::mutex m;
    unsigned char* base = nullptr;
    int64_t slot = 0; // bytes per slot; 2 slots per thread
    unsigned char* slots(int64_t slot_bytes)
    {
        if (base && slot >= slot_bytes) return base;
        if (base) cudaFreeHost(base);
        base = nullptr;
        void* p = nullptr;
        SDFO_CUDA(cudaHostAlloc(&p, (size_t)(2 * kMaxThreads * slot_bytes),
                                cudaHostAllocPortable | cudaHostAllocMapped));
        base = static_cast<unsigned char*>(p);
        slot = slot_bytes;
        return base;
    }
};

PinnedPool& pool()
{
    static PinnedPool* p = new PinnedPool(); // never destroyed: outlives static teardown
    return *p;
}

// One contiguous piece of a transfer: `bytes` at file offset `off` to / from
// device memory `dev`, or (dev NULL) block records `first` .. `first+count-1`
// that a kernel decodes from / packs into the pinned slot.
struct Chunk
{
    int64_t off;
    int64_t bytes;
    unsigned char* dev;
    int64_t first;
    int64_t count;
};

// Splits [off, off + bytes) -> dev into pieces of at most `max_bytes`.
void split(std::vector<Chunk>& out, int64_t off, int64_t bytes, void* dev, int64_t max_bytes)
{
    unsigned char* d = static_cast<unsigned char*>(dev);
    for (int64_t k = 0; k < bytes; k += max_bytes)
        out.push_back({off + k, std::min(max_bytes, bytes - k), d + k, -1, 0});
}

// A worker's view of its two pinned slots: host addresses and the device
// addresses of the same memory.
struct Slots
{
    unsigned char* h[2];
    unsigned char* d[2];
};

struct Workers
{
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> done;
    cudaEvent_t start = nullptr;
    ~Workers()
    {
        for (auto e : done) cudaEventDestroy(e);
        for (auto st : streams) cudaStreamDestroy(st);
        if (start) cudaEventDestroy(start);
    }
};

using WorkFn = std::function<void(int t, cudaStream_t st, const Slots& sl)>;

// Runs `work` on T threads (thread 0 is the calling thread), each with its
// own stream ordered after everything already on `s`; `s` then waits for all
// of them and is synchronised.  The first error of any thread is rethrown.
void run_workers(int T, cudaStream_t s, int64_t slot_bytes, const WorkFn& work)
{
    unsigned char* host = pool().slots(slot_bytes);
    void* dev = nullptr;
    SDFO_CUDA(cudaHostGetDevicePointer(&dev, host, 0));
    Workers w;
    SDFO_CUDA(cudaEventCreateWithFlags(&w.start, cudaEventDisableTiming));
    SDFO_CUDA(cudaEventRecord(w.start, s));
    for (int t = 0; t < T; ++t)
    {
        cudaStream_t st;
        SDFO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        w.streams.push_back(st);
        cudaEvent_t e;
        SDFO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        w.done.push_back(e);
        SDFO_CUDA(cudaStreamWaitEvent(st, w.start, 0));
    }
    std::vector<Error> errs(T, Error(SDFO_OK, ""));
    auto body = [&](int t) {
        Slots sl;
        for (int k = 0; k < 2; ++k)
        {
            const int64_t off = (2 * t + k) * slot_bytes;
            sl.h[k] = host + off;
            sl.d[k] = static_cast<unsigned char*>(dev) + off;
        }
        try
        {
            work(t, w.streams[t], sl);
        }
        catch (const Error& e)
        {
            errs[t] = e;
        }
        catch (const std::exception& e)
        {
            errs[t] = Error(SDFO_ERR_IO, e.what());
        }
        cudaEventRecord(w.done[t], w.streams[t]);
    };
    std::vector<std::thread> th;
    for (int t = 1; t < T; ++t) th.emplace_back(body, t);
    body(0);
    for (auto& x : th) x.join();
    for (int t = 0; t < T; ++t) SDFO_CUDA(cudaStreamWaitEvent(s, w.done[t], 0));
    SDFO_CUDA(cudaStreamSynchronize(s));
    for (int t = 0; t < T; ++t)
        if (errs[t].code != SDFO_OK) throw errs[t];
}

int pick_threads(size_t chunks)
{
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    return (int)std::max<size_t>(1, std::min<size_t>({(size_t)kMaxThreads, (size_t)hw, (chunks + 1) / 2}));
}

struct SlotEvents
{
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t st;
    explicit SlotEvents(cudaStream_t s) : st(s)
    {
        SDFO_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
        SDFO_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
    }
    ~SlotEvents()
    {
        cudaStreamSynchronize(st); // nothing may still use the slots
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    }
};

using RecordFn = std::function<void(const Chunk&, unsigned char* d_slot, cudaStream_t)>;

// File -> device: thread t takes chunks t, t+T, ...; pread into one pinned
// slot while the other slot's copy (or decoding kernel) runs.
void load_chunks(int fd, const std::vector<Chunk>& chunks, cudaStream_t s, int64_t slot_bytes,
                 const RecordFn& decode)
{
    if (chunks.empty()) return;
    const int T = pick_threads(chunks.size());
    run_workers(T, s, slot_bytes, [&](int t, cudaStream_t st, const Slots& sl) {
        SlotEvents e(st);
        bool pending[2] = {false, false};
        int use = 0;
        for (size_t k = (size_t)t; k < chunks.size(); k += (size_t)T)
        {
            const Chunk& c = chunks[k];
            if (pending[use]) SDFO_CUDA(cudaEventSynchronize(e.ev[use]));
            if (pread_full(fd, sl.h[use], c.bytes, c.off) != c.bytes) io_error("short read");
            if (c.dev)
                SDFO_CUDA(cudaMemcpyAsync(c.dev, sl.h[use], (size_t)c.bytes, cudaMemcpyHostToDevice, st));
            else
                decode(c, sl.d[use], st);
            SDFO_CUDA(cudaEventRecord(e.ev[use], st));
            pending[use] = true;
            use ^= 1;
        }
    });
}

// Device -> file: the copy (or packing kernel) of chunk k+T is in flight
// while chunk k is written.
void put_chunk(const File& f, const void* src, int64_t bytes, int64_t off);

void save_chunks(const File& f, const std::vector<Chunk>& chunks, cudaStream_t s, int64_t slot_bytes,
                 const RecordFn& pack)
{
    if (chunks.empty()) return;
    const int T = pick_threads(chunks.size());
    run_workers(T, s, slot_bytes, [&](int t, cudaStream_t st, const Slots& sl) {
        SlotEvents e(st);
        auto issue = [&](size_t k, int slot) {
            const Chunk& c = chunks[k];
            if (c.dev)
                SDFO_CUDA(cudaMemcpyAsync(sl.h[slot], c.dev, (size_t)c.bytes, cudaMemcpyDeviceToHost, st));
            else
                pack(c, sl.d[slot], st);
            SDFO_CUDA(cudaEventRecord(e.ev[slot], st));
        };
        int use = 0;
        if ((size_t)t < chunks.size()) issue((size_t)t, 0);
        for (size_t k = (size_t)t; k < chunks.size(); k += (size_t)T)
        {
            if (k + (size_t)T < chunks.size()) issue(k + (size_t)T, use ^ 1);
            SDFO_CUDA(cudaEventSynchronize(e.ev[use]));
            put_chunk(f, sl.h[use], chunks[k].bytes, chunks[k].off);
            use ^= 1;
        }
    });
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
constexpr int kThreads = 256;

unsigned grid_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, 148 * 16)); }

template <class T>
__device__ __forceinline__ T load_any(const unsigned char* p)
{
    T v;
    if ((reinterpret_cast<uintptr_t>(p) & (sizeof(T) - 1)) == 0)
        v = *reinterpret_cast<const T*>(p);
    else
    {
        unsigned char* q = reinterpret_cast<unsigned char*>(&v);
#pragma unroll
        for (int i = 0; i < (int)sizeof(T); ++i) q[i] = p[i];
    }
    return v;
}

template <class T>
__device__ __forceinline__ void store_any(unsigned char* p, T v)
{
    if ((reinterpret_cast<uintptr_t>(p) & (sizeof(T) - 1)) == 0)
        *reinterpret_cast<T*>(p) = v;
    else
    {
        const unsigned char* q = reinterpret_cast<const unsigned char*>(&v);
#pragma unroll
        for (int i = 0; i < (int)sizeof(T); ++i) p[i] = q[i];
    }
}

// Dense: FP32 {phi, n} payload and FP32 Hessians from the FP64 arrays.
__global__ void k_dense_decode(const double* __restrict__ phi, const double* __restrict__ n,
                               const double* __restrict__ h, int64_t N, float4* __restrict__ phin,
                               float* __restrict__ hess6)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    {
        phin[i] = make_float4((float)phi[i], (float)n[3 * i], (float)n[3 * i + 1], (float)n[3 * i + 2]);
        if (h)
        {
#pragma unroll
            for (int k = 0; k < 6; ++k) hess6[6 * i + k] = (float)h[6 * i + k];
        }
    }
}

// Dense candidate counts: u32 in the file, u8 on the device; the first index
// whose count exceeds the stride goes to *bad.
__global__ void k_counts_u32_to_u8(const uint32_t* __restrict__ c32, int64_t N, int s,
                                   uint8_t* __restrict__ c8, unsigned long long* bad)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    {
        const uint32_t c = c32[i];
        if (c > (uint32_t)s) atomicMin(bad, (unsigned long long)i);
        c8[i] = (uint8_t)(c > 255u ? 255u : c);
    }
}

__global__ void k_counts_u8_to_u32(const uint8_t* __restrict__ c8, int64_t N, uint32_t* __restrict__ c32)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
        c32[i] = c8[i];
}

// Dense export sources for grids without FP64 arrays: phi / n from the FP32
// payload, Hessians from the FP32 ones.
__global__ void k_dense_fp64_from_payload(const float4* __restrict__ phin, const float* __restrict__ hess6,
                                          int64_t N, double* __restrict__ phi, double* __restrict__ n,
                                          double* __restrict__ h)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    {
        const float4 v = phin[i];
        if (phi) phi[i] = v.x;
        if (n)
        {
            n[3 * i] = v.y;
            n[3 * i + 1] = v.z;
            n[3 * i + 2] = v.w;
        }
        if (h)
        {
#pragma unroll
            for (int k = 0; k < 6; ++k) h[6 * i + k] = hess6 ? (double)hess6[6 * i + k] : 0.0;
        }
    }
}

// Byte layout of one sparse block record (SdfIO.cpp:226-272).
struct Record
{
    int V, s, has_h;
    int64_t bytes;
    int64_t off_phi, off_n, off_h, off_cnt, off_cphi, off_cn, off_cbr;
};

Record record_layout(int bd, int has_h, int s)
{
    Record r;
    r.V = bd * bd * bd;
    r.s = s;
    r.has_h = has_h;
    const int64_t V = r.V;
    r.off_phi = kBlockHeaderBytes;
    r.off_n = r.off_phi + 4 * V;
    r.off_h = r.off_n + 12 * V;
    r.off_cnt = r.off_h + (has_h ? 24 * V : 0);
    r.off_cphi = r.off_cnt + (s ? V : 0);
    r.off_cn = r.off_cphi + 4 * V * s;
    r.off_cbr = r.off_cn + 12 * V * s;
    r.bytes = r.off_cbr + 4 * V * s;
    return r;
}

struct SparseArrays
{
    int32_t* ijk;
    float4* phin;
    float* hess6;
    uint8_t* ca_count;
    float* ca_phi;
    float* ca_n;
    int32_t* ca_branch;
    // FP16 sources for saving
    const ushort4* phin16;
    const float2* affine;
};

// One CTA per record of the chunk: the record's header, {phi, n} (interleaved
// into float4), Hessians and candidates.
__global__ void __launch_bounds__(kThreads) k_sparse_decode(const unsigned char* __restrict__ raw, Record r,
                                                           int64_t first, SparseArrays a,
                                                           unsigned long long* bad_block)
{
    const int64_t b = first + blockIdx.x;
    const unsigned char* rec = raw + (int64_t)blockIdx.x * r.bytes;
    const int64_t V = r.V;
    if (threadIdx.x < 3) a.ijk[3 * b + threadIdx.x] = load_any<int32_t>(rec + 4 * threadIdx.x);
    for (int64_t v = threadIdx.x; v < V; v += blockDim.x)
    {
        const float p = load_any<float>(rec + r.off_phi + 4 * v);
        const float x = load_any<float>(rec + r.off_n + 12 * v);
        const float y = load_any<float>(rec + r.off_n + 12 * v + 4);
        const float z = load_any<float>(rec + r.off_n + 12 * v + 8);
        a.phin[b * V + v] = make_float4(p, x, y, z);
    }
    if (r.has_h)
        for (int64_t i = threadIdx.x; i < 6 * V; i += blockDim.x)
            a.hess6[b * 6 * V + i] = load_any<float>(rec + r.off_h + 4 * i);
    if (r.s)
    {
        const int64_t M = V * r.s;
        bool bad = false;
        for (int64_t v = threadIdx.x; v < V; v += blockDim.x)
        {
            const uint8_t c = rec[r.off_cnt + v];
            bad = bad || c > r.s;
            a.ca_count[b * V + v] = c;
        }
        if (bad) atomicMin(bad_block, (unsigned long long)b);
        for (int64_t i = threadIdx.x; i < M; i += blockDim.x)
        {
            a.ca_phi[b * M + i] = load_any<float>(rec + r.off_cphi + 4 * i);
            a.ca_branch[b * M + i] = load_any<int32_t>(rec + r.off_cbr + 4 * i);
        }
        for (int64_t i = threadIdx.x; i < 3 * M; i += blockDim.x)
            a.ca_n[b * 3 * M + i] = load_any<float>(rec + r.off_cn + 4 * i);
    }
}

// The inverse of k_sparse_decode (FP16 payloads decoded to FP32 as the
// export does).
__global__ void __launch_bounds__(kThreads) k_sparse_pack(unsigned char* __restrict__ raw, Record r, int64_t first,
                                                         SparseArrays a)
{
    const int64_t b = first + blockIdx.x;
    unsigned char* rec = raw + (int64_t)blockIdx.x * r.bytes;
    const int64_t V = r.V;
    if (threadIdx.x < 4) store_any<int32_t>(rec + 4 * threadIdx.x, threadIdx.x < 3 ? a.ijk[3 * b + threadIdx.x] : 0);
    for (int64_t v = threadIdx.x; v < V; v += blockDim.x)
    {
        float4 q;
        if (a.phin16)
        {
            const ushort4 h = a.phin16[b * V + v];
            const float2 af = a.affine[b];
            q = make_float4(__fadd_rn(__fmul_rn(__half2float(__ushort_as_half(h.x)), af.x), af.y),
                            __half2float(__ushort_as_half(h.y)),
                            __half2float(__ushort_as_half(h.z)), __half2float(__ushort_as_half(h.w)));
        }
        else
            q = a.phin[b * V + v];
        store_any<float>(rec + r.off_phi + 4 * v, q.x);
        store_any<float>(rec + r.off_n + 12 * v, q.y);
        store_any<float>(rec + r.off_n + 12 * v + 4, q.z);
        store_any<float>(rec + r.off_n + 12 * v + 8, q.w);
    }
    if (r.has_h)
        for (int64_t i = threadIdx.x; i < 6 * V; i += blockDim.x)
            store_any<float>(rec + r.off_h + 4 * i, a.hess6 ? a.hess6[b * 6 * V + i] : 0.f);
    if (r.s)
    {
        const int64_t M = V * r.s;
        for (int64_t v = threadIdx.x; v < V; v += blockDim.x) rec[r.off_cnt + v] = a.ca_count[b * V + v];
        for (int64_t i = threadIdx.x; i < M; i += blockDim.x)
        {
            store_any<float>(rec + r.off_cphi + 4 * i, a.ca_phi[b * M + i]);
            store_any<int32_t>(rec + r.off_cbr + 4 * i, a.ca_branch[b * M + i]);
        }
        for (int64_t i = threadIdx.x; i < 3 * M; i += blockDim.x)
            store_any<float>(rec + r.off_cn + 4 * i, a.ca_n[b * 3 * M + i]);
    }
}

constexpr int32_t kNoBlock = 0x7f7f7f7f; // cudaMemset(0x7f) of an int32 table

// Block table: the lowest block index per coordinate (first wins), blocks
// outside the grid's block range are unreachable by in-grid voxels and skipped.
__global__ void k_table_claim(const int32_t* __restrict__ ijk, int64_t B, int nbx, int nby, int nbz,
                              int32_t* table)
{
    for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < B; b += (int64_t)gridDim.x * blockDim.x)
    {
        const int bi = ijk[3 * b], bj = ijk[3 * b + 1], bk = ijk[3 * b + 2];
        if (bi < 0 || bj < 0 || bk < 0 || bi >= nbx || bj >= nby || bk >= nbz) continue;
        atomicMin(table + (bi + (int64_t)nbx * (bj + (int64_t)nby * bk)), (int32_t)b);
    }
}

__global__ void k_table_finish(int32_t* table, int64_t T)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T; i += (int64_t)gridDim.x * blockDim.x)
        if (table[i] == kNoBlock) table[i] = -1;
}

// ---------------------------------------------------------------------------
// load
// ---------------------------------------------------------------------------
void open_for_read(File& f, const char* path)
{
    f.fd = ::open(path, O_RDONLY | O_CLOEXEC);
    if (f.fd < 0) io_error(std::string("Cannot open SdfOracle data file: ") + path);
    struct stat st;
    if (::fstat(f.fd, &st) != 0) io_error(std::string("Cannot open SdfOracle data file: ") + path);
    f.size = (int64_t)st.st_size;
}

Header read_checked_header(const File& f)
{
    unsigned char b[kHeaderBytes];
    if (pread_full(f.fd, b, kHeaderBytes, 0) != kHeaderBytes) io_error("Failed to read SdfOracle data header");
    Header h = parse_header(b);
    if (std::memcmp(h.magic, "SDFO", 4) != 0) io_error("Invalid SdfOracle data magic number");
    if (h.version != kVersion)
        io_error("Unsupported SdfOracle data version: " + std::to_string(h.version) +
                 " (only 0.1.0 is supported)");
    return h;
}

bool header_is_sparse(const Header& h)
{
    const uint32_t layout = get_u32(h.reserved, 0);
    return (h.flags & kFlagSparse) != 0 && (layout == kLayoutSparse || layout == kLayoutCaSparse);
}

sdfo_grid_info info_from_header(const Header& h)
{
    sdfo_grid_info info{};
    const uint32_t n[3] = {h.nx, h.ny, h.nz};
    for (int a = 0; a < 3; ++a)
    {
        info.bmin[a] = h.bmin[a];
        info.bmax[a] = h.bmax[a];
        info.voxel[a] = h.voxel[a];
        SDFO_REQUIRE(n[a] > 0 && n[a] <= (uint32_t)INT32_MAX, SDFO_ERR_UNSUPPORTED,
                     "SDFO grid shape must be positive");
        info.shape[a] = (int32_t)n[a];
        SDFO_REQUIRE(h.voxel[a] > 0.0 && std::isfinite(h.voxel[a]) && std::isfinite(h.bmin[a]),
                     SDFO_ERR_UNSUPPORTED, "SDFO grid spec must have finite bmin and positive voxel size");
    }
    const int64_t N = (int64_t)info.shape[0] * info.shape[1] * info.shape[2];
    SDFO_REQUIRE(N < (int64_t(1) << 40), SDFO_ERR_UNSUPPORTED, "grid too large");
    info.storage = SDFO_STORAGE_FP32;
    return info;
}

// loadSdf (SdfIO.cpp:277-380).
sdfo_grid* load_dense(const File& f, const Header& h, cudaStream_t s)
{
    if (h.flags & kFlagSparse) io_error("SdfOracle data file uses sparse layout; call loadSparseSdf");
    const uint32_t layout = get_u32(h.reserved, 0);
    if (layout != kLayoutDense && layout != kLayoutCaDense)
        io_error("SdfOracle data file is not dense 0.1.0 layout");
    const bool ca_flag = (h.flags & kFlagCandidates) != 0;
    if ((layout == kLayoutCaDense) != ca_flag) io_error("Dense SDF 0.1.0 contact-aware flag/layout mismatch");
    const bool has_ca = ca_flag && layout == kLayoutCaDense;
    const bool has_h = (h.flags & kFlagHessian) != 0;

    sdfo_grid_info info = info_from_header(h);
    info.layout = SDFO_LAYOUT_DENSE;
    info.has_hessian = has_h ? 1 : 0;
    const int64_t N = (int64_t)info.shape[0] * info.shape[1] * info.shape[2];
    int s_ca = 0;
    if (has_ca)
    {
        s_ca = (int)get_u32(h.reserved, 4);
        if (s_ca <= 0 || s_ca > kMaxCandidates) io_error("Invalid contact-aware candidate stride");
    }

    Laps tm;
    std::unique_ptr<sdfo_grid> g(new sdfo_grid());
    g->info = info;
    g->stored_voxels = N;
    SDFO_CUDA(cudaGetDevice(&g->device));
    g->d.phin = dalloc<float4>((size_t)N);
    g->d.phi64 = dalloc<double>((size_t)N);
    g->d.n64 = dalloc<double>((size_t)N * 3);
    g->d.w64 = dalloc<double>((size_t)N * 3);
    if (has_h)
    {
        g->d.h64 = dalloc<double>((size_t)N * 6);
        g->d.hess6 = dalloc<float>((size_t)N * 6);
    }
    DeviceBuffer<uint32_t> c32;
    if (has_ca)
    {
        const int64_t M = N * s_ca;
        c32.reset((size_t)N);
        SDFO_CUDA(cudaMemsetAsync(c32.get(), 0, sizeof(uint32_t) * N, s));
        g->d.ca_count = dalloc<uint8_t>((size_t)N);
        g->d.ca_phi64 = dalloc<double>((size_t)M);
        g->d.ca_n64 = dalloc<double>((size_t)M * 3);
        g->d.ca_branch = dalloc<int32_t>((size_t)M);
    }

    // sections in file order, clipped at the end of the file
    struct Section
    {
        void* dev;
        int64_t bytes;
    };
    std::vector<Section> sec = {{g->d.phi64, 8 * N}, {g->d.n64, 24 * N}};
    if (has_h) sec.push_back({g->d.h64, 48 * N});
    sec.push_back({g->d.w64, 24 * N});
    if (has_ca)
    {
        const int64_t M = N * s_ca;
        sec.push_back({c32.get(), 4 * N});
        sec.push_back({g->d.ca_phi64, 8 * M});
        sec.push_back({g->d.ca_n64, 24 * M});
        sec.push_back({g->d.ca_branch, 4 * M});
    }
    std::vector<Chunk> chunks;
    int64_t off = kHeaderBytes;
    bool truncated = false;
    for (size_t i = 0; i < sec.size(); ++i)
    {
        const int64_t avail = std::max<int64_t>(0, std::min(sec[i].bytes, f.size - off));
        if (avail < sec[i].bytes) truncated = true;
        // a clipped counts section keeps only whole entries
        const int64_t take = (has_ca && sec[i].dev == c32.get()) ? avail / 4 * 4 : avail;
        split(chunks, off, take, sec[i].dev, kSlotBytes);
        off += sec[i].bytes;
    }
    g->stats.setup_ms = tm.lap();
    load_chunks(f.fd, chunks, s, kSlotBytes, nullptr);
    g->stats.fill_ms = tm.lap();
    if (has_ca)
    {
        DeviceBuffer<unsigned long long> bad(1);
        SDFO_CUDA(cudaMemsetAsync(bad.get(), 0xff, sizeof(unsigned long long), s));
        k_counts_u32_to_u8<<<grid_for(N), kThreads, 0, s>>>(c32.get(), N, s_ca, g->d.ca_count, bad.get());
        SDFO_CHECK_LAUNCH();
        unsigned long long hb = 0;
        SDFO_CUDA(cudaMemcpyAsync(&hb, bad.get(), sizeof(hb), cudaMemcpyDeviceToHost, s));
        SDFO_CUDA(cudaStreamSynchronize(s));
        if (hb != ~0ull) io_error("Invalid contact-aware candidate count");
        g->ca_stride = s_ca;
        g->info.candidate_stride = s_ca;
    }
    if (truncated) io_error("Failed to read dense SDF payload");
    k_dense_decode<<<grid_for(N), kThreads, 0, s>>>(g->d.phi64, g->d.n64, g->d.h64, N, g->d.phin, g->d.hess6);
    SDFO_CHECK_LAUNCH();
    build_stencil_layouts(g.get(), s);
    SDFO_CUDA(cudaStreamSynchronize(s));
    g->stats.hessian_ms = tm.lap();
    g->stats.total_ms = tm.total();
    g->stats.voxels_filled = N;
    return g.release();
}

// loadSparseSdf (SdfIO.cpp:382-523).
sdfo_grid* load_sparse(const File& f, const Header& h, cudaStream_t s)
{
    const uint32_t layout = get_u32(h.reserved, 0);
    const bool ca_flag = (h.flags & kFlagCandidates) != 0;
    if ((layout == kLayoutCaSparse) != ca_flag) io_error("Sparse SDF 0.1.0 contact-aware flag/layout mismatch");
    const bool has_ca = ca_flag && layout == kLayoutCaSparse;
    if ((h.flags & kFlagSparse) == 0 || !(layout == kLayoutSparse || has_ca))
        io_error("SdfOracle data file is not sparse block 0.1.0");
    const int bd = (int)get_u32(h.reserved, 4);
    const int halo = (int)get_u32(h.reserved, 8);
    const uint32_t block_count = get_u32(h.reserved, 12);
    const double band = get_f64(h.reserved, 16);
    const bool has_h = (h.flags & kFlagHessian) != 0;
    const int s_ca = has_ca ? (int)get_u32(h.reserved, 24) : 0;
    if (bd <= 0) io_error("Sparse SDF blockDim must be positive");
    if (has_ca && (s_ca <= 0 || s_ca > kMaxCandidates)) io_error("Invalid sparse contact-aware candidate stride");
    SDFO_REQUIRE(bd <= 64, SDFO_ERR_UNSUPPORTED, "sparse blockDim above 64 is not supported");
    SDFO_REQUIRE(block_count < (uint32_t)kNoBlock, SDFO_ERR_UNSUPPORTED, "too many sparse blocks");

    sdfo_grid_info info = info_from_header(h);
    info.layout = SDFO_LAYOUT_SPARSE;
    info.has_hessian = has_h ? 1 : 0;
    info.block_dim = bd;
    info.halo_voxels = halo;
    info.band_distance = band;
    const Record r = record_layout(bd, has_h ? 1 : 0, s_ca);
    const int64_t V = r.V;

    // whole records present in the file; the first partial one decides the
    // error the reference would raise for it
    const int64_t body = std::max<int64_t>(0, f.size - kHeaderBytes);
    const int64_t complete = std::min<int64_t>((int64_t)block_count, body / r.bytes);
    const int64_t B = complete;

    Laps tm;
    std::unique_ptr<sdfo_grid> g(new sdfo_grid());
    g->info = info;
    g->info.block_count = (int32_t)B;
    SDFO_CUDA(cudaGetDevice(&g->device));
    for (int a = 0; a < 3; ++a) g->nb[a] = (info.shape[a] + bd - 1) / bd;
    g->stored_voxels = B * V;
    const int64_t T = (int64_t)g->nb[0] * g->nb[1] * g->nb[2];
    g->d.table = dalloc<int32_t>((size_t)T);
    SparseArrays a{};
    if (B > 0)
    {
        g->d.ijk = dalloc<int32_t>((size_t)B * 3);
        g->d.phin = dalloc<float4>((size_t)(B * V));
        if (has_h) g->d.hess6 = dalloc<float>((size_t)(B * V * 6));
        if (has_ca)
        {
            const int64_t M = B * V * s_ca;
            g->d.ca_count = dalloc<uint8_t>((size_t)(B * V));
            g->d.ca_phi32 = dalloc<float>((size_t)M);
            g->d.ca_n32 = dalloc<float>((size_t)M * 3);
            g->d.ca_branch = dalloc<int32_t>((size_t)M);
        }
        a = SparseArrays{g->d.ijk, g->d.phin, g->d.hess6, g->d.ca_count, g->d.ca_phi32, g->d.ca_n32, g->d.ca_branch,
                         nullptr, nullptr};
    }
    DeviceBuffer<unsigned long long> bad(1);
    SDFO_CUDA(cudaMemsetAsync(bad.get(), 0xff, sizeof(unsigned long long), s));
    const int64_t per_chunk = std::max<int64_t>(1, kSlotBytes / r.bytes);
    const int64_t slot_bytes = std::max<int64_t>(kSlotBytes, r.bytes);
    std::vector<Chunk> chunks;
    for (int64_t b = 0; b < B; b += per_chunk)
    {
        const int64_t nb = std::min(per_chunk, B - b);
        chunks.push_back({kHeaderBytes + b * r.bytes, nb * r.bytes, nullptr, b, nb});
    }
    unsigned long long* d_bad = bad.get();
    g->stats.setup_ms = tm.lap();
    load_chunks(f.fd, chunks, s, slot_bytes, [&](const Chunk& c, unsigned char* d_slot, cudaStream_t st) {
                    k_sparse_decode<<<(unsigned)c.count, kThreads, 0, st>>>(d_slot, r, c.first, a, d_bad);
                    SDFO_CHECK_LAUNCH();
                });
    unsigned long long hb = 0;
    SDFO_CUDA(cudaMemcpyAsync(&hb, d_bad, sizeof(hb), cudaMemcpyDeviceToHost, s));
    SDFO_CUDA(cudaStreamSynchronize(s));
    if (hb != ~0ull) io_error("Invalid sparse contact-aware candidate count");
    g->stats.fill_ms = tm.lap();
    if (B < (int64_t)block_count)
    {
        // the record after the last complete one is cut short
        const int64_t off = kHeaderBytes + B * r.bytes;
        const int64_t avail = std::max<int64_t>(0, f.size - off);
        if (avail < kBlockHeaderBytes) io_error("Failed to read sparse SDF block header");
        if (has_ca && avail > r.off_cnt)
        {
            std::vector<uint8_t> cnt((size_t)std::min<int64_t>(V, avail - r.off_cnt));
            pread_full(f.fd, cnt.data(), (int64_t)cnt.size(), off + r.off_cnt);
            for (uint8_t c : cnt)
                if (c > s_ca) io_error("Invalid sparse contact-aware candidate count");
        }
        io_error("Failed to read sparse SDF block payload");
    }
    SDFO_CUDA(cudaMemsetAsync(g->d.table, 0x7f, sizeof(int32_t) * T, s));
    if (B > 0)
    {
        k_table_claim<<<grid_for(B), kThreads, 0, s>>>(g->d.ijk, B, g->nb[0], g->nb[1], g->nb[2], g->d.table);
        SDFO_CHECK_LAUNCH();
    }
    k_table_finish<<<grid_for(T), kThreads, 0, s>>>(g->d.table, T);
    SDFO_CHECK_LAUNCH();
    if (has_ca)
    {
        g->ca_stride = s_ca;
        g->info.candidate_stride = s_ca;
    }
    build_stencil_layouts(g.get(), s);
    SDFO_CUDA(cudaStreamSynchronize(s));
    g->stats.hessian_ms = tm.lap();
    g->stats.total_ms = tm.total();
    g->stats.voxels_filled = B * V;
    return g.release();
}

// ---------------------------------------------------------------------------
// save
// ---------------------------------------------------------------------------
// Opens, sizes and (where the file system can preallocate it, so that a full
// disk is reported here and not as a fault on a mapped store) maps the output
// file: the worker threads then copy chunks into the mapping in parallel,
// which scales where concurrent pwrite() calls on one file serialise on its
// inode lock.  Without preallocation the chunks are written with pwrite().
void open_for_write(File& f, const char* path, int64_t size)
{
    f.fd = ::open(path, O_RDWR | O_CREAT | O_TRUNC | O_CLOEXEC, 0666);
    if (f.fd < 0) io_error(std::string("Cannot open SdfOracle data file for writing: ") + path);
    if (::ftruncate(f.fd, (off_t)size) != 0)
        io_error(std::string("Failed to write SdfOracle data file: ") + std::strerror(errno));
    f.size = size;
    if (size <= 0) return;
    // fallocate(2) itself, not posix_fallocate, whose fallback writes zeros
    if (::fallocate(f.fd, 0, 0, (off_t)size) != 0)
    {
        if (errno == ENOSPC || errno == EFBIG)
            io_error(std::string("Failed to write SdfOracle data file: ") + std::strerror(errno));
        return; // no preallocation on this file system: pwrite
    }
    void* m = ::mmap(nullptr, (size_t)size, PROT_READ | PROT_WRITE, MAP_SHARED, f.fd, 0);
    if (m != MAP_FAILED) f.map = static_cast<unsigned char*>(m);
}

// Writes one chunk's bytes at its file offset.
void put_chunk(const File& f, const void* src, int64_t bytes, int64_t off)
{
    if (f.map)
        std::memcpy(f.map + off, src, (size_t)bytes);
    else
        pwrite_full(f.fd, src, bytes, off);
}

// saveSdf (SdfIO.cpp:93-174): header, phi, n, H (always), witness, candidates.
void save_dense(const sdfo_grid* g, const char* path, cudaStream_t s)
{
    const int64_t N = g->stored_voxels;
    const int sc = g->ca_stride;
    const int64_t M = N * sc;
    DeviceBuffer<double> t_phi, t_n, t_h, t_w;
    const double* phi = g->d.phi64;
    const double* n = g->d.n64;
    const double* h = g->d.h64;
    const double* w = g->d.w64;
    if (!phi || !n || !h)
    {
        if (!phi) t_phi.reset((size_t)N);
        if (!n) t_n.reset((size_t)N * 3);
        if (!h) t_h.reset((size_t)N * 6);
        k_dense_fp64_from_payload<<<grid_for(N), kThreads, 0, s>>>(g->d.phin, g->d.hess6, N, t_phi.get(), t_n.get(),
                                                                  t_h.get());
        SDFO_CHECK_LAUNCH();
        if (!phi) phi = t_phi.get();
        if (!n) n = t_n.get();
        if (!h) h = t_h.get();
    }
    if (!w)
    {
        t_w.reset((size_t)N * 3);
        SDFO_CUDA(cudaMemsetAsync(t_w.get(), 0, sizeof(double) * 3 * N, s));
        w = t_w.get();
    }
    DeviceBuffer<uint32_t> c32;
    if (sc)
    {
        c32.reset((size_t)N);
        k_counts_u8_to_u32<<<grid_for(N), kThreads, 0, s>>>(g->d.ca_count, N, c32.get());
        SDFO_CHECK_LAUNCH();
    }
    std::vector<std::pair<const void*, int64_t>> sec = {{phi, 8 * N}, {n, 24 * N}, {h, 48 * N}, {w, 24 * N}};
    if (sc)
    {
        sec.push_back({c32.get(), 4 * N});
        sec.push_back({g->d.ca_phi64, 8 * M});
        sec.push_back({g->d.ca_n64, 24 * M});
        sec.push_back({g->d.ca_branch, 4 * M});
    }
    int64_t total = kHeaderBytes;
    for (auto& x : sec) total += x.second;
    unsigned char hdr[kHeaderBytes];
    write_header(hdr, g->info, kFlagHessian | (sc ? kFlagCandidates : 0u));
    put_u32(hdr + 96, 0, sc ? kLayoutCaDense : kLayoutDense);
    if (sc) put_u32(hdr + 96, 4, (uint32_t)sc);
    File f;
    open_for_write(f, path, total);
    put_chunk(f, hdr, kHeaderBytes, 0);
    std::vector<Chunk> chunks;
    int64_t off = kHeaderBytes;
    for (auto& x : sec)
    {
        split(chunks, off, x.second, const_cast<void*>(x.first), kSlotBytes);
        off += x.second;
    }
    save_chunks(f, chunks, s, kSlotBytes, nullptr);
    if (!f.finish()) io_error("Failed to write SdfOracle data file");
}

// saveSparseSdf (SdfIO.cpp:176-275): header, then per block its record.
void save_sparse(const sdfo_grid* g, const char* path, cudaStream_t s)
{
    const int bd = g->info.block_dim;
    SDFO_REQUIRE(bd > 0, SDFO_ERR_IO, "Sparse SDF blockDim must be positive");
    const int64_t B = g->info.block_count;
    const int sc = g->ca_stride;
    const bool has_h = g->info.has_hessian != 0;
    const Record r = record_layout(bd, has_h ? 1 : 0, sc);
    unsigned char hdr[kHeaderBytes];
    write_header(hdr, g->info, kFlagSparse | (has_h ? kFlagHessian : 0u) | (sc ? kFlagCandidates : 0u));
    put_u32(hdr + 96, 0, sc ? kLayoutCaSparse : kLayoutSparse);
    put_u32(hdr + 96, 4, (uint32_t)bd);
    put_u32(hdr + 96, 8, (uint32_t)g->info.halo_voxels);
    put_u32(hdr + 96, 12, (uint32_t)B);
    put_f64(hdr + 96, 16, g->info.band_distance);
    if (sc) put_u32(hdr + 96, 24, (uint32_t)sc);
    File f;
    open_for_write(f, path, kHeaderBytes + B * r.bytes);
    put_chunk(f, hdr, kHeaderBytes, 0);
    const SparseArrays a{g->d.ijk, g->d.phin, g->d.hess6, g->d.ca_count, g->d.ca_phi32, g->d.ca_n32, g->d.ca_branch,
                         g->info.storage == SDFO_STORAGE_FP16 ? g->d.phin16 : nullptr,
                         g->info.storage == SDFO_STORAGE_FP16 ? g->d.brick_affine : nullptr};
    const int64_t per_chunk = std::max<int64_t>(1, kSlotBytes / r.bytes);
    const int64_t slot_bytes = std::max<int64_t>(kSlotBytes, r.bytes);
    std::vector<Chunk> chunks;
    for (int64_t b = 0; b < B; b += per_chunk)
    {
        const int64_t nb = std::min(per_chunk, B - b);
        chunks.push_back({kHeaderBytes + b * r.bytes, nb * r.bytes, nullptr, b, nb});
    }
    save_chunks(f, chunks, s, slot_bytes, [&](const Chunk& c, unsigned char* d_slot, cudaStream_t st) {
                    k_sparse_pack<<<(unsigned)c.count, kThreads, 0, st>>>(d_slot, r, c.first, a);
                    SDFO_CHECK_LAUNCH();
                });
    if (!f.finish()) io_error("Failed to write SdfOracle data file");
}

} // namespace
} // namespace sdfo

using namespace sdfo;

extern "C" {

int sdfo_file_probe(const char* path, int32_t* is_valid, int32_t* is_sparse)
{
    return guarded([&] {
        SDFO_REQUIRE(path != nullptr, SDFO_ERR_INVALID_ARGUMENT, "path is NULL");
        if (is_valid) *is_valid = 0;
        if (is_sparse) *is_sparse = 0;
        const int fd = ::open(path, O_RDONLY | O_CLOEXEC);
        if (fd < 0) return;
        unsigned char b[kHeaderBytes];
        const int64_t got = pread_full(fd, b, kHeaderBytes, 0);
        ::close(fd);
        if (got != kHeaderBytes) return;
        const Header h = parse_header(b);
        const bool valid = std::memcmp(h.magic, "SDFO", 4) == 0 && h.version == kVersion;
        if (is_valid) *is_valid = valid ? 1 : 0;
        if (is_sparse) *is_sparse = valid && header_is_sparse(h) ? 1 : 0;
    });
}

int sdfo_grid_load_file(const char* path, int32_t expect, void* stream, sdfo_grid** out)
{
    return guarded([&] {
        SDFO_REQUIRE(path && out, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        SDFO_REQUIRE(expect >= SDFO_FILE_ANY && expect <= SDFO_FILE_SPARSE, SDFO_ERR_INVALID_ARGUMENT,
                     "expect must be SDFO_FILE_ANY, SDFO_FILE_DENSE or SDFO_FILE_SPARSE");
        *out = nullptr;
        File f;
        open_for_read(f, path);
        const Header h = read_checked_header(f);
        bool sparse = expect == SDFO_FILE_SPARSE;
        if (expect == SDFO_FILE_ANY) sparse = header_is_sparse(h);
        std::lock_guard<std::mutex> lock(pool().m);
        cudaStream_t s = as_stream(stream);
        *out = sparse ? load_sparse(f, h, s) : load_dense(f, h, s);
    });
}

int sdfo_grid_save_file(const sdfo_grid* g, const char* path, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(g && path, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        std::lock_guard<std::mutex> lock(pool().m);
        cudaStream_t s = as_stream(stream);
        if (g->info.layout == SDFO_LAYOUT_SPARSE)
            save_sparse(g, path, s);
        else
            save_dense(g, path, s);
    });
}

} // extern "C"
