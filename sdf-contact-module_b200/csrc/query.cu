// Batched SDF query kernels (forward, forward-mode Jacobian, backward).
//
// One thread per query point.  A query reads its point (12 or 24 B, streamed
// with evict-first loads), gathers the 8 cell corners as one 16-B {phi, n}
// vector load each (dense: x-fastest voxel array; sparse: block table lookup
// then brick payload), evaluates the interpolant in FP32 and streams out
// gap, raw gradient, unit normal, witness, valid flag and optionally the
// 3x3 Hessian (the Jacobian of the gradient w.r.t. the point).
//
// Reference behaviour reproduced: SdfOracle::queryFast and the per-mode
// queries (SdfOracle.cpp:226-432, 448-851, 932-1092): invalid when any
// corner is outside the grid or (sparse) its block is not stored; unit normal
// falls back to UnitX when |grad| <= 1e-15 (SecondOrder: to n0).
#include "bulk.cuh"
#include "interp.cuh"

#include <algorithm>
#include <atomic>
#include <mutex>

namespace sdfo {
namespace {

constexpr int kThreads = 256;

template <typename PT>
__device__ __forceinline__ void load_point(const PT* pts, int64_t q, double p[3])
{
    p[0] = (double)__ldcs(pts + 3 * q + 0);
    p[1] = (double)__ldcs(pts + 3 * q + 1);
    p[2] = (double)__ldcs(pts + 3 * q + 2);
}

// Block-cooperative I/O of K-float records (points in; gradient, unit,
// witness, Hessian out): the block's 256 records are one contiguous range,
// moved with 16-byte accesses through shared memory instead of K 4-byte
// accesses per thread at a 4K-byte stride.  Used when the pointers are
// 16-byte aligned (the host checks); `src`/`dst` point at the block's first
// record and `cnt` = records of this block.
template <int K>
__device__ __forceinline__ void stage_in(float* sbuf, const float* src, int cnt)
{
    const int nf = K * cnt, nv = nf >> 2;
    for (int t = threadIdx.x; t < nv; t += kThreads)
        reinterpret_cast<float4*>(sbuf)[t] = __ldcs(reinterpret_cast<const float4*>(src) + t);
    for (int t = 4 * nv + threadIdx.x; t < nf; t += kThreads) sbuf[t] = __ldcs(src + t);
}

template <int K>
__device__ __forceinline__ void stage_out(const float* sbuf, float* dst, int cnt)
{
    const int nf = K * cnt, nv = nf >> 2;
    for (int t = threadIdx.x; t < nv; t += kThreads)
        __stcs(reinterpret_cast<float4*>(dst) + t, reinterpret_cast<const float4*>(sbuf)[t]);
    for (int t = 4 * nv + threadIdx.x; t < nf; t += kThreads) __stcs(dst + t, sbuf[t]);
}

// This thread's K-float record of a block-uniform array (staged or direct).
template <int K, bool STAGED>
__device__ __forceinline__ void read_rec(float* sbuf, const float* base, int64_t q0, int cnt,
                                         bool active, float r[K])
{
    if (STAGED)
    {
        __syncthreads();
        stage_in<K>(sbuf, base + K * q0, cnt);
        __syncthreads();
#pragma unroll
        for (int a = 0; a < K; ++a) r[a] = active ? sbuf[K * threadIdx.x + a] : 0.f;
    }
    else
    {
#pragma unroll
        for (int a = 0; a < K; ++a) r[a] = active ? __ldcs(base + K * (q0 + threadIdx.x) + a) : 0.f;
    }
}

template <int K, bool STAGED>
__device__ __forceinline__ void write_rec(float* sbuf, float* base, int64_t q0, int cnt,
                                          bool active, const float r[K])
{
    if (STAGED)
    {
        __syncthreads();
#pragma unroll
        for (int a = 0; a < K; ++a) sbuf[K * threadIdx.x + a] = r[a];
        __syncthreads();
        stage_out<K>(sbuf, base + K * q0, cnt);
    }
    else if (active)
    {
#pragma unroll
        for (int a = 0; a < K; ++a) __stcs(base + K * (q0 + threadIdx.x) + a, r[a]);
    }
}

// dL/d(stored payload) of one valid query: the interpolant is linear in
// the corner values, so the scatter weights are the basis functions (and
// their derivatives / h for the gradient outputs) at the point.  float4
// atomics {d phi, d n} per corner.  A corner whose brick is not stored
// (possible only when the caller's valid flags belong to other points or
// another grid) is skipped.
template <int MODE, bool SPARSE, int BD>
__device__ __forceinline__ void scatter_grid_gradient(const GridView& g, const Cell& c, float dG,
                                                      const float dg[3], float* dgrid)
{
    const float h[3] = {(float)g.voxel[0], (float)g.voxel[1], (float)g.voxel[2]};
    const float ig[3] = {dg[0] * g.ih[0], dg[1] * g.ih[1], dg[2] * g.ih[2]};
    float4* out = reinterpret_cast<float4*>(dgrid);
    auto index = [&](int k) -> int64_t {
        const int i = c.i0 + (k & 1), j = c.j0 + ((k >> 1) & 1), kk = c.k0 + (k >> 2);
        return SPARSE ? sparse_index<BD>(g, i, j, kk) : dense_index(g, i, j, kk);
    };
    if (MODE == SDFO_TRICUBIC)
    {
        float bx[4], dx[4], by[4], dy[4], bz[4], dz[4];
        hermite(c.u, bx, dx);
        hermite(c.v, by, dy);
        hermite(c.w, bz, dz);
#pragma unroll
        for (int k = 0; k < 8; ++k)
        {
            const int di = k & 1, dj = (k >> 1) & 1, dk = k >> 2;
            const float P0 = bx[2 * di], P1 = bx[2 * di + 1], dP0 = dx[2 * di], dP1 = dx[2 * di + 1];
            const float Q0 = by[2 * dj], Q1 = by[2 * dj + 1], dQ0 = dy[2 * dj], dQ1 = dy[2 * dj + 1];
            const float R0 = bz[2 * dk], R1 = bz[2 * dk + 1], dR0 = dz[2 * dk], dR1 = dz[2 * dk + 1];
            // d/d phi_k
            const float wphi = dG * (P0 * Q0 * R0) + ig[0] * (dP0 * Q0 * R0) +
                               ig[1] * (P0 * dQ0 * R0) + ig[2] * (P0 * Q0 * dR0);
            // d/d (n h) components, chained through the slope n * h
            const float wgx = dG * (P1 * Q0 * R0) + ig[0] * (dP1 * Q0 * R0) +
                              ig[1] * (P1 * dQ0 * R0) + ig[2] * (P1 * Q0 * dR0);
            const float wgy = dG * (P0 * Q1 * R0) + ig[0] * (dP0 * Q1 * R0) +
                              ig[1] * (P0 * dQ1 * R0) + ig[2] * (P0 * Q1 * dR0);
            const float wgz = dG * (P0 * Q0 * R1) + ig[0] * (dP0 * Q0 * R1) +
                              ig[1] * (P0 * dQ0 * R1) + ig[2] * (P0 * Q0 * dR1);
            const int64_t ix = index(k);
            if (ix >= 0) atomicAdd(out + ix, make_float4(wphi, wgx * h[0], wgy * h[1], wgz * h[2]));
        }
    }
    else
    {
        const float u = c.u, v = c.v, w = c.w;
        const float bu[2] = {1.f - u, u}, bv[2] = {1.f - v, v}, bw[2] = {1.f - w, w};
        const float du[2] = {-1.f, 1.f};
#pragma unroll
        for (int k = 0; k < 8; ++k)
        {
            const int di = k & 1, dj = (k >> 1) & 1, dk = k >> 2;
            const float wphi = dG * (bu[di] * bv[dj] * bw[dk]) + ig[0] * (du[di] * bv[dj] * bw[dk]) +
                               ig[1] * (bu[di] * du[dj] * bw[dk]) + ig[2] * (bu[di] * bv[dj] * du[dk]);
            const int64_t ix = index(k);
            if (ix >= 0) atomicAdd(&out[ix].x, wphi);
        }
    }
}

// Minimum resident CTAs per SM requested from the register allocator for
// the plain query and for the query with the Hessian.
#ifndef SDFO_QUERY_MIN_BLOCKS
#define SDFO_QUERY_MIN_BLOCKS 5
#endif
// Sparse gathers: 4 CTAs per SM (64 registers) measured faster than 5 (48
// registers, with spills) and 6 on the 512^3 icosphere: FP32 23.8 against
// 23.2 and 17.2 G queries/s, FP16 20.7 against 19.5 and 14.8.
#ifndef SDFO_QUERY_SPARSE_MIN_BLOCKS
#define SDFO_QUERY_SPARSE_MIN_BLOCKS 4
#endif
#ifndef SDFO_QUERY_HESS_MIN_BLOCKS
#define SDFO_QUERY_HESS_MIN_BLOCKS 4
#endif
template <bool HESS, bool SPARSE = false>
constexpr int query_min_blocks()
{
    return HESS ? SDFO_QUERY_HESS_MIN_BLOCKS : SPARSE ? SDFO_QUERY_SPARSE_MIN_BLOCKS : SDFO_QUERY_MIN_BLOCKS;
}

template <int MODE, bool SPARSE, int BD, typename PT, bool HESS, bool STAGED>
__global__ void __launch_bounds__(kThreads, query_min_blocks<HESS, SPARSE>())
    k_query(GridView g, const PT* __restrict__ pts, int64_t n, QueryOutputs o)
{
    __shared__ __align__(16) float sbuf[STAGED ? (HESS ? 6 : 3) * kThreads : 1];
    const int64_t q0 = (int64_t)blockIdx.x * kThreads;
    const int64_t q = q0 + threadIdx.x;
    const bool active = q < n;
    const int cnt = (int)(n - q0 < kThreads ? n - q0 : kThreads);
    double p[3] = {0.0, 0.0, 0.0};
    if (STAGED)
    {
        float pf[3];
        read_rec<3, true>(sbuf, reinterpret_cast<const float*>(pts), q0, cnt, active, pf);
        p[0] = pf[0];
        p[1] = pf[1];
        p[2] = pf[2];
    }
    else if (active)
    {
        load_point(pts, q, p);
    }
    Interp r;
    float unit[3] = {1.f, 0.f, 0.f};
    const bool want_unit = o.unit != nullptr || o.witness != nullptr;
    const bool valid = active && evaluate<MODE, SPARSE, BD, HESS>(g, p, r, unit, want_unit);
    if (!valid)
    {
        r.gap = 0.f;
        r.g[0] = r.g[1] = r.g[2] = 0.f;
        unit[0] = 1.f;
        unit[1] = unit[2] = 0.f;
#pragma unroll
        for (int a = 0; a < 6; ++a) r.H[a] = 0.f;
    }
    if (active)
    {
        __stcs(o.gap + q, r.gap);
        if (o.valid) o.valid[q] = valid ? 1 : 0;
    }
    // the output pointers are uniform over the block
    if (o.grad) write_rec<3, STAGED>(sbuf, o.grad, q0, cnt, active, r.g);
    if (o.unit) write_rec<3, STAGED>(sbuf, o.unit, q0, cnt, active, unit);
    if (o.witness)
    {
        float w[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) w[a] = valid ? (float)(p[a] - (double)r.gap * unit[a]) : 0.f;
        write_rec<3, STAGED>(sbuf, o.witness, q0, cnt, active, w);
    }
    if (HESS && o.hess6) write_rec<6, STAGED>(sbuf, o.hess6, q0, cnt, active, r.H);
    if (HESS && o.hess && active)
    {
        const float H9[9] = {r.H[0], r.H[1], r.H[2], r.H[1], r.H[3], r.H[4], r.H[2], r.H[4], r.H[5]};
#pragma unroll
        for (int a = 0; a < 9; ++a) __stcs(o.hess + 9 * q + a, H9[a]);
    }
}

// Persistent variant of k_query for FP32 points (sparse grids: every output;
// dense grids: without the Hessian): CTA c walks the contiguous tile range
// [ntiles c / G, ntiles (c + 1) / G) of kThreads queries (measured 10%
// faster than grid-stride order on random points over one grid; points
// sorted in space stay coherent within a CTA's range).  Each
// thread loads the point of its next tile before it evaluates the current
// one, and loads and stores go straight to global memory, so warps never wait
// for one another (k_query stages points and records through shared memory
// between CTA barriers).  Selected by sdfo_tuning.query_walk.
// Records of K floats of a warp's 32 consecutive queries q0 .. q0 + cnt - 1,
// stored through the warp's slice of shared memory (32 K floats): each lane
// writes its record, then the warp writes the slice out as contiguous 16-byte
// stores (a full warp) or contiguous 4-byte stores (the tail of the last
// tile).  Without this, each of a lane's K strided 4-byte stores touches K
// cache lines per warp instruction.  `direct`: the output is not 16-byte
// aligned; each lane stores its record itself.
template <int K>
__device__ __forceinline__ void warp_store(float* __restrict__ slice, float* __restrict__ out, int64_t q0,
                                           int cnt, const float v[K], bool direct)
{
    const int lane = (int)(threadIdx.x & 31);
    if (direct)
    {
        if (lane < cnt)
#pragma unroll
            for (int a = 0; a < K; ++a) __stcs(out + K * (q0 + lane) + a, v[a]);
        return;
    }
#pragma unroll
    for (int a = 0; a < K; ++a) slice[K * lane + a] = v[a];
    __syncwarp();
    float* dst = out + K * q0;
    if (cnt == 32)
    {
        // 32 K floats = 8 K float4, at a 16-byte aligned address (q0 is a
        // multiple of 32)
        const float4* src = reinterpret_cast<const float4*>(slice);
        for (int i = lane; i < 8 * K; i += 32) __stcs(reinterpret_cast<float4*>(dst) + i, src[i]);
    }
    else
    {
        for (int i = lane; i < K * cnt; i += 32) __stcs(dst + i, slice[i]);
    }
    __syncwarp(); // the slice is rewritten by the next tile
}

template <int MODE, bool SPARSE, int BD, bool HESS, int MINB, int ST>
__global__ void __launch_bounds__(kThreads, MINB)
    k_query_walk(GridView g, const float* __restrict__ pts, int64_t n, QueryOutputs o)
{
    // Hessian records (6 or 9 floats) leave through per-warp slices
    __shared__ __align__(16) float stage[HESS ? kThreads * 9 : 1];
    const int64_t ntiles = (n + kThreads - 1) / kThreads;
    const int64_t t_begin = ntiles * blockIdx.x / gridDim.x;
    const int64_t t_end = ntiles * (blockIdx.x + 1) / gridDim.x;
    int64_t q = t_begin * kThreads + threadIdx.x;
    float xn[3] = {0.f, 0.f, 0.f};
    if (t_begin < t_end && q < n)
        for (int a = 0; a < 3; ++a) xn[a] = __ldcs(pts + 3 * q + a);
    const bool want_unit = o.unit != nullptr || o.witness != nullptr;
    const int lane = (int)(threadIdx.x & 31);
    float* slice = stage + (HESS ? (threadIdx.x >> 5) * 32 * 9 : 0);
    const bool h6_direct = (reinterpret_cast<uintptr_t>(o.hess6) & 15) != 0;
    const bool h9_direct = (reinterpret_cast<uintptr_t>(o.hess) & 15) != 0;
    for (int64_t t = t_begin; t < t_end; ++t)
    {
        const int64_t qc = q;
        const double p[3] = {xn[0], xn[1], xn[2]};
        q += kThreads;
        if (t + 1 < t_end && q < n)
            for (int a = 0; a < 3; ++a) xn[a] = __ldcs(pts + 3 * q + a);
        // the tail of the last tile: lanes past n skip the work but (HESS)
        // still take part in their warp's staged stores
        const bool live = qc < n;
        if (!HESS && !live) continue;
        Interp r;
        float unit[3] = {1.f, 0.f, 0.f};
        const bool valid = live && evaluate<MODE, SPARSE, BD, HESS, ST>(g, p, r, unit, want_unit);
        if (!valid)
        {
            r.gap = 0.f;
            r.g[0] = r.g[1] = r.g[2] = 0.f;
            unit[0] = 1.f;
            unit[1] = unit[2] = 0.f;
#pragma unroll
            for (int a = 0; a < 6; ++a) r.H[a] = 0.f;
        }
        if (live)
        {
            __stcs(o.gap + qc, r.gap);
            if (o.valid) o.valid[qc] = valid ? 1 : 0;
            if (o.grad)
                for (int a = 0; a < 3; ++a) __stcs(o.grad + 3 * qc + a, r.g[a]);
            if (o.unit)
                for (int a = 0; a < 3; ++a) __stcs(o.unit + 3 * qc + a, unit[a]);
            if (o.witness)
                for (int a = 0; a < 3; ++a)
                    __stcs(o.witness + 3 * qc + a, valid ? (float)(p[a] - (double)r.gap * unit[a]) : 0.f);
        }
        if constexpr (HESS)
        {
            // warp-uniform: the warp's first query and how many of its 32 exist
            const int64_t qw = qc - lane;
            const int64_t left = n - qw;
            const int cnt = left >= 32 ? 32 : (left > 0 ? (int)left : 0);
            if (o.hess6) warp_store<6>(slice, o.hess6, qw, cnt, r.H, h6_direct);
            if (o.hess)
            {
                const float H9[9] = {r.H[0], r.H[1], r.H[2], r.H[1], r.H[3], r.H[4], r.H[2], r.H[4], r.H[5]};
                warp_store<9>(slice, o.hess, qw, cnt, H9, h9_direct);
            }
        }
    }
}

template <int MODE, bool SPARSE, int BD, bool HESS, int MINB, int ST = 0>
void launch_walk(const GridView& v, const float* pts, int64_t n, const QueryOutputs& o, cudaStream_t s)
{
    static std::mutex mu;
    static int per_sm[64] = {0};
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    int b;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (per_sm[dev & 63] == 0)
        {
            int r = 0;
            SDFO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_query_walk<MODE, SPARSE, BD, HESS, MINB, ST>, kThreads, 0));
            per_sm[dev & 63] = r > 0 ? r : 1;
        }
        b = per_sm[dev & 63];
    }
    const int64_t ntiles = (n + kThreads - 1) / kThreads;
    const unsigned blocks = (unsigned)std::min<int64_t>(ntiles, (int64_t)current_sm_count() * b);
    k_query_walk<MODE, SPARSE, BD, HESS, MINB, ST><<<blocks, kThreads, 0, s>>>(v, pts, n, o);
}

// Reverse mode from the linearisation the forward saved (grad, symmetric
// Hessian, valid flag): dL/dp = dgap * grad + H dgrad is elementwise, and the
// grid gradient needs only the corner weights, which depend on the point
// but not on the grid values, so nothing of the grid is read again.
template <int MODE, bool SPARSE, int BD, bool STAGED, bool DPTS, bool DGRID>
__global__ void __launch_bounds__(kThreads)
    k_backward_saved(GridView g, const float* __restrict__ pts, int64_t n,
                     const float* __restrict__ grad, const float* __restrict__ hess6,
                     const uint8_t* __restrict__ valid, const float* __restrict__ dgap,
                     const float* __restrict__ dgrad, float* __restrict__ dpts,
                     float* __restrict__ dgrid)
{
    // staged inputs, all loaded before one barrier: dgrad | grad | hess6
    __shared__ __align__(16) float sbuf[STAGED ? 12 * kThreads : 1];
    const int64_t q0 = (int64_t)blockIdx.x * kThreads;
    const int64_t q = q0 + threadIdx.x;
    const bool active = q < n;
    const int cnt = (int)(n - q0 < kThreads ? n - q0 : kThreads);
    const float dG = (dgap && active) ? __ldcs(dgap + q) : 0.f;
    float dg[3] = {0.f, 0.f, 0.f};
    if (DPTS)
    {
        float gr[3] = {0.f, 0.f, 0.f}, H[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (STAGED)
        {
            if (dgrad) stage_in<3>(sbuf, dgrad + 3 * q0, cnt);
            stage_in<3>(sbuf + 3 * kThreads, grad + 3 * q0, cnt);
            stage_in<6>(sbuf + 6 * kThreads, hess6 + 6 * q0, cnt);
            __syncthreads();
            if (active)
            {
#pragma unroll
                for (int a = 0; a < 3; ++a)
                {
                    if (dgrad) dg[a] = sbuf[3 * threadIdx.x + a];
                    gr[a] = sbuf[3 * kThreads + 3 * threadIdx.x + a];
                }
#pragma unroll
                for (int a = 0; a < 6; ++a) H[a] = sbuf[6 * kThreads + 6 * threadIdx.x + a];
            }
        }
        else if (active)
        {
#pragma unroll
            for (int a = 0; a < 3; ++a)
            {
                if (dgrad) dg[a] = __ldcs(dgrad + 3 * q + a);
                gr[a] = __ldcs(grad + 3 * q + a);
            }
#pragma unroll
            for (int a = 0; a < 6; ++a) H[a] = __ldcs(hess6 + 6 * q + a);
        }
        const float out[3] = {dG * gr[0] + H[0] * dg[0] + H[1] * dg[1] + H[2] * dg[2],
                              dG * gr[1] + H[1] * dg[0] + H[3] * dg[1] + H[4] * dg[2],
                              dG * gr[2] + H[2] * dg[0] + H[4] * dg[1] + H[5] * dg[2]};
        write_rec<3, STAGED>(sbuf, dpts, q0, cnt, active, out);
    }
    else if (dgrad)
    {
        read_rec<3, STAGED>(sbuf, dgrad, q0, cnt, active, dg);
    }
    if (DGRID)
    {
        float pf[3];
        read_rec<3, STAGED>(sbuf, pts, q0, cnt, active, pf);
        if (!active || !valid[q]) return;
        const double p[3] = {pf[0], pf[1], pf[2]};
        const Cell c = cell_of(g, p);
        if (!c.ok) return;
        scatter_grid_gradient<MODE, SPARSE, BD>(g, c, dG, dg, dgrid);
    }
}

// Backward with the stencil gathered again (no saved state): dL/dp =
// dgap * grad + H dgrad, and the grid gradient scatter.
template <int MODE, bool SPARSE, int BD>
__global__ void __launch_bounds__(kThreads)
    k_query_backward(GridView g, const float* __restrict__ pts, int64_t n,
                     const float* __restrict__ dgap, const float* __restrict__ dgrad,
                     float* __restrict__ dpts, float* __restrict__ dgrid)
{
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= n) return;
    double p[3];
    load_point(pts, q, p);
    const float dG = dgap ? __ldcs(dgap + q) : 0.f;
    float dg[3] = {0.f, 0.f, 0.f};
    if (dgrad)
    {
        dg[0] = __ldcs(dgrad + 3 * q + 0);
        dg[1] = __ldcs(dgrad + 3 * q + 1);
        dg[2] = __ldcs(dgrad + 3 * q + 2);
    }
    Interp r;
    float unit[3];
    const bool ok = evaluate<MODE, SPARSE, BD, true>(g, p, r, unit);
    if (dpts)
    {
        const float* H = r.H;
#pragma unroll
        for (int a = 0; a < 3; ++a) dpts[3 * q + a] = 0.f;
        if (ok)
        {
            dpts[3 * q + 0] = dG * r.g[0] + H[0] * dg[0] + H[1] * dg[1] + H[2] * dg[2];
            dpts[3 * q + 1] = dG * r.g[1] + H[1] * dg[0] + H[3] * dg[1] + H[4] * dg[2];
            dpts[3 * q + 2] = dG * r.g[2] + H[2] * dg[0] + H[4] * dg[1] + H[5] * dg[2];
        }
    }
    if (!dgrid || !ok) return;
    scatter_grid_gradient<MODE, SPARSE, BD>(g, cell_of(g, p), dG, dg, dgrid);
}

// Persistent variant of k_query_backward (sdfo_tuning.query_walk): CTA c
// walks the contiguous tile range [ntiles c / G, ntiles (c + 1) / G) of
// kThreads queries, and each thread loads the next tile's point and upstream
// gradients before it regathers the current one.
template <int MODE, bool SPARSE, int BD, int ST, bool DGRID>
__global__ void __launch_bounds__(kThreads, 3)
    k_query_backward_walk(GridView g, const float* __restrict__ pts, int64_t n,
                          const float* __restrict__ dgap, const float* __restrict__ dgrad,
                          float* __restrict__ dpts, float* __restrict__ dgrid)
{
    const int64_t ntiles = (n + kThreads - 1) / kThreads;
    const int64_t t_begin = ntiles * blockIdx.x / gridDim.x;
    const int64_t t_end = ntiles * (blockIdx.x + 1) / gridDim.x;
    int64_t q = t_begin * kThreads + threadIdx.x;
    float xn[3] = {0.f, 0.f, 0.f}, dGn = 0.f, dgn[3] = {0.f, 0.f, 0.f};
    auto fetch = [&](int64_t i) {
        for (int a = 0; a < 3; ++a) xn[a] = __ldcs(pts + 3 * i + a);
        if (dgap) dGn = __ldcs(dgap + i);
        if (dgrad)
            for (int a = 0; a < 3; ++a) dgn[a] = __ldcs(dgrad + 3 * i + a);
    };
    if (t_begin < t_end && q < n) fetch(q);
    for (int64_t t = t_begin; t < t_end; ++t)
    {
        const int64_t qc = q;
        const double p[3] = {xn[0], xn[1], xn[2]};
        const float dG = dGn;
        const float dg[3] = {dgn[0], dgn[1], dgn[2]};
        q += kThreads;
        if (t + 1 < t_end && q < n) fetch(q);
        if (qc >= n) continue; // the tail of the last tile
        Interp r;
        float unit[3];
        const bool ok = evaluate<MODE, SPARSE, BD, true, ST>(g, p, r, unit, false);
        if (dpts)
        {
            const float* H = r.H;
            float o3[3] = {0.f, 0.f, 0.f};
            if (ok)
            {
                o3[0] = dG * r.g[0] + H[0] * dg[0] + H[1] * dg[1] + H[2] * dg[2];
                o3[1] = dG * r.g[1] + H[1] * dg[0] + H[3] * dg[1] + H[4] * dg[2];
                o3[2] = dG * r.g[2] + H[2] * dg[0] + H[4] * dg[1] + H[5] * dg[2];
            }
            for (int a = 0; a < 3; ++a) __stcs(dpts + 3 * qc + a, o3[a]);
        }
        if (DGRID && ok) scatter_grid_gradient<MODE, SPARSE, BD>(g, cell_of(g, p), dG, dg, dgrid);
    }
}

template <int MODE, bool SPARSE, int BD, int ST, bool DGRID>
void launch_bwd_walk2(const GridView& v, const float* pts, int64_t n, const float* dgap, const float* dgrad,
                     float* dpts, float* dgrid, cudaStream_t s)
{
    static std::mutex mu;
    static int per_sm[64] = {0};
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    int b;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (per_sm[dev & 63] == 0)
        {
            int r = 0;
            SDFO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                &r, k_query_backward_walk<MODE, SPARSE, BD, ST, DGRID>, kThreads, 0));
            per_sm[dev & 63] = r > 0 ? r : 1;
        }
        b = per_sm[dev & 63];
    }
    const int64_t ntiles = (n + kThreads - 1) / kThreads;
    const unsigned blocks = (unsigned)std::min<int64_t>(ntiles, (int64_t)current_sm_count() * b);
    k_query_backward_walk<MODE, SPARSE, BD, ST, DGRID><<<blocks, kThreads, 0, s>>>(v, pts, n, dgap, dgrad, dpts,
                                                                                 dgrid);
}

// points only: the walk with the grid-gradient scatter needs more than 80
// registers (100-250 bytes of spills), so that backward keeps the per-tile
// kernel
template <int MODE, bool SPARSE, int BD, int ST>
void launch_bwd_walk(const GridView& v, const float* pts, int64_t n, const float* dgap, const float* dgrad,
                     float* dpts, cudaStream_t s)
{
    launch_bwd_walk2<MODE, SPARSE, BD, ST, false>(v, pts, n, dgap, dgrad, dpts, nullptr, s);
}

template <int MODE, bool SPARSE, int BD, bool HESS>
void launch_pt2(const GridView& v, const void* pts, bool f64, bool staged, int64_t n,
                const QueryOutputs& o, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
    if (f64)
        k_query<MODE, SPARSE, BD, double, HESS, false><<<blocks, kThreads, 0, s>>>(
            v, static_cast<const double*>(pts), n, o);
    else if (staged)
        k_query<MODE, SPARSE, BD, float, HESS, true><<<blocks, kThreads, 0, s>>>(
            v, static_cast<const float*>(pts), n, o);
    else
        k_query<MODE, SPARSE, BD, float, HESS, false><<<blocks, kThreads, 0, s>>>(
            v, static_cast<const float*>(pts), n, o);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

std::atomic<bool> g_query_walk{true};

} // namespace

bool query_walk() { return g_query_walk.load(); }
void set_query_walk(bool on) { g_query_walk.store(on); }

namespace {

// Persistent, bulk-copy-pipelined variant of k_query for FP32 points on dense
// grids and the outputs gap, raw gradient, valid flag and (HESS) the
// symmetric Hessian:
// each CTA walks tiles of kThreads queries; point tiles arrive by
// cp.async.bulk three tiles ahead (so no query waits on its point load), the
// output tiles are written to shared memory and leave by bulk stores.  The
// last n mod kThreads points take plain loads and stores in the last CTA,
// which takes no tile.  Bounded waits, as in stream_bwd.cu (status bit 1 when
// one runs out).
constexpr int kPipeStages = 3;
constexpr unsigned kPipeWaitLimit = 1u << 24;
__device__ unsigned int g_pipe_status = 0;
// Test-only: {main-loop wait limit (0 = kPipeWaitLimit), withhold the first
// tile's load in every CTA}; both 0 in normal operation.
__device__ unsigned int g_pipe_test[2] = {0u, 0u};

template <bool HESS>
struct PipeLayout
{
    static constexpr int pts = 12 * kThreads;                        // one stage
    static constexpr int gap = 4 * kThreads, grad = 12 * kThreads, valid = kThreads;
    static constexpr int hess = HESS ? 24 * kThreads : 0;
    static constexpr int out = gap + grad + valid + hess;            // one output buffer
    static constexpr int total = kPipeStages * pts + 2 * out;
};

template <int MODE, bool SPARSE, int BD, bool HESS>
__global__ void __launch_bounds__(kThreads, query_min_blocks<HESS>())
    k_query_pipe(GridView g, const float* __restrict__ pts, int64_t n, QueryOutputs o)
{
    using L = PipeLayout<HESS>;
    using namespace bulk;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bars[kPipeStages];
    __shared__ int s_abort;
    __shared__ long long s_kabort;
    __shared__ unsigned s_limit;
    __shared__ int s_withhold;
    unsigned char* stages = smem;
    unsigned char* outs = smem + kPipeStages * L::pts;
    const int64_t tiles = n / kThreads;
    // with a remainder the last CTA takes it (plain loads and stores) and
    // leaves; the others walk the whole tiles
    const bool rem = (n % kThreads) != 0;
    if (rem && blockIdx.x == gridDim.x - 1)
    {
        const int64_t q = tiles * kThreads + threadIdx.x;
        if (q >= n) return;
        const double p[3] = {pts[3 * q], pts[3 * q + 1], pts[3 * q + 2]};
        Interp r;
        float unit[3];
        const bool valid = evaluate<MODE, SPARSE, BD, HESS>(g, p, r, unit, false);
        if (!valid)
        {
            r.gap = 0.f;
            r.g[0] = r.g[1] = r.g[2] = 0.f;
#pragma unroll
            for (int a = 0; a < 6; ++a) r.H[a] = 0.f;
        }
        o.gap[q] = r.gap;
        if (o.grad)
            for (int a = 0; a < 3; ++a) o.grad[3 * q + a] = r.g[a];
        if (o.valid) o.valid[q] = valid ? 1 : 0;
        if (HESS && o.hess6)
            for (int a = 0; a < 6; ++a) o.hess6[6 * q + a] = r.H[a];
        return;
    }
    const int64_t first = blockIdx.x, step = gridDim.x - (rem ? 1 : 0);
    const int64_t mine = first < tiles ? (tiles - first + step - 1) / step : 0;
    if (threadIdx.x == 0)
    {
        s_abort = 0;
        s_limit = g_pipe_test[0] ? g_pipe_test[0] : kPipeWaitLimit;
        s_withhold = g_pipe_test[1] != 0u;
        for (int st = 0; st < kPipeStages; ++st) mbar_init(&bars[st], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int k = 0; k < kPipeStages && k < mine; ++k)
        {
            if (k == 0 && s_withhold) continue; // test: tile 0's barrier never completes
            mbar_expect_tx(&bars[k], L::pts);
            bulk_load(stages + k * L::pts, pts + 3 * (first + k * step) * kThreads, L::pts, &bars[k]);
        }
    }
    __syncthreads();
    for (int64_t k = 0; k < mine; ++k)
    {
        const int st = (int)(k % kPipeStages);
        const unsigned parity = (unsigned)((k / kPipeStages) & 1);
        unsigned it = 0;
        while (!mbar_try_wait(&bars[st], parity))
            if (++it >= s_limit)
            {
                s_abort = 1;
                s_kabort = k;
                break;
            }
        __syncthreads();
        if (s_abort) break;
        const float* pf = reinterpret_cast<const float*>(stages + st * L::pts) + 3 * threadIdx.x;
        const double p[3] = {pf[0], pf[1], pf[2]};
        Interp r;
        float unit[3];
        const bool valid = evaluate<MODE, SPARSE, BD, HESS>(g, p, r, unit, false);
        if (!valid)
        {
            r.gap = 0.f;
            r.g[0] = r.g[1] = r.g[2] = 0.f;
#pragma unroll
            for (int a = 0; a < 6; ++a) r.H[a] = 0.f;
        }
        unsigned char* ob = outs + (int)(k & 1) * L::out;
        if (threadIdx.x == 0 && k >= 2) bulk_wait_read<1>(); // the stores of tile k-2 have read this buffer
        __syncthreads();
        reinterpret_cast<float*>(ob)[threadIdx.x] = r.gap;
        float* gr = reinterpret_cast<float*>(ob + L::gap) + 3 * threadIdx.x;
        gr[0] = r.g[0];
        gr[1] = r.g[1];
        gr[2] = r.g[2];
        ob[L::gap + L::grad + threadIdx.x] = valid ? 1 : 0;
        if (HESS)
        {
            float* h6 = reinterpret_cast<float*>(ob + L::gap + L::grad + L::valid) + 6 * threadIdx.x;
#pragma unroll
            for (int a = 0; a < 6; ++a) h6[a] = r.H[a];
        }
        fence_async_shared();
        __syncthreads(); // stage st consumed, outputs written
        if (threadIdx.x == 0)
        {
            const int64_t q0 = (first + k * step) * kThreads;
            bulk_store(o.gap + q0, ob, L::gap);
            if (o.grad) bulk_store(o.grad + 3 * q0, ob + L::gap, L::grad);
            if (o.valid) bulk_store(o.valid + q0, ob + L::gap + L::grad, L::valid);
            if (HESS && o.hess6) bulk_store(o.hess6 + 6 * q0, ob + L::gap + L::grad + L::valid, L::hess);
            bulk_commit();
            const int64_t nk = k + kPipeStages;
            if (nk < mine)
            {
                mbar_expect_tx(&bars[st], L::pts);
                bulk_load(stages + st * L::pts, pts + 3 * (first + nk * step) * kThreads, L::pts, &bars[st]);
            }
        }
    }
    if (threadIdx.x == 0)
    {
        if (s_abort)
        {
            atomicOr(&g_pipe_status, kPipeStatusWaitAbort);
            // the tiles issued but not consumed complete into this CTA's
            // shared memory: wait for them (bounded, the full limit) before
            // the CTA exits; a withheld tile has nothing in flight
            for (long long j = s_kabort; j < s_kabort + kPipeStages && j < mine; ++j)
            {
                if (j == 0 && s_withhold) continue;
                unsigned it = 0;
                while (!mbar_try_wait(&bars[j % kPipeStages], (unsigned)((j / kPipeStages) & 1)) &&
                       ++it < kPipeWaitLimit)
                {
                }
            }
        }
        bulk_wait_read<0>();
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
}

// A float32 query through k_query_pipe when the outputs allow it (gap, grad,
// valid, hess6 only; 16-byte aligned) and there is at least one whole tile;
// returns whether it was taken.
template <int MODE, bool SPARSE, int BD>
bool launch_pipe(const GridView& v, const float* pts, int64_t n, const QueryOutputs& o, cudaStream_t s)
{
    if (n < kThreads || o.host_mapped || o.unit || o.witness || o.hess || !o.gap || !aligned16(pts) || !aligned16(o.gap) ||
        !aligned16(o.grad) || !aligned16(o.valid) || !aligned16(o.hess6))
        return false;
    const int sms = current_sm_count();
    const int64_t tiles = n / kThreads;
    const int64_t rem = n % kThreads ? 1 : 0; // one more CTA, for the remainder
    if (o.hess6)
    {
        const int64_t ctas = std::min<int64_t>(tiles, (int64_t)sms * query_min_blocks<true>() - rem) + rem;
        k_query_pipe<MODE, SPARSE, BD, true>
            <<<(unsigned)ctas, kThreads, PipeLayout<true>::total, s>>>(v, pts, n, o);
    }
    else
    {
        const int64_t ctas = std::min<int64_t>(tiles, (int64_t)sms * query_min_blocks<false>() - rem) + rem;
        k_query_pipe<MODE, SPARSE, BD, false>
            <<<(unsigned)ctas, kThreads, PipeLayout<false>::total, s>>>(v, pts, n, o);
    }
    SDFO_CHECK_LAUNCH();
    return true;
}

template <int MODE, bool SPARSE, int BD>
void launch_pt(const GridView& v, const void* pts, bool f64, int64_t n, const QueryOutputs& o, cudaStream_t s)
{
    // The persistent walk (query_walk(), the default) for FP32 points and
    // results in device memory (results in mapped host memory take the staged
    // kernel, whose 16-byte accesses suit the bus).  Register budgets
    // (resident CTAs per SM) measured on the hollow cylinder (dense) and the
    // 512^3 icosphere (sparse):
    //   dense, no Hessian: 4 CTAs (64 registers, no spills), 32.5 G queries/s
    //     against 28.7 for the bulk-copy pipeline;
    //   dense, full 3x3 Hessian: 3 CTAs, 25.8 G/s against 17.1 for the staged
    //     kernel (the pipeline writes only the 6 unique entries);
    //   dense, 6-entry Hessian (the linearising forward): stays on the
    //     pipeline -- as a walk it ran 24.4-26.4 against 25.7 G/s, but the
    //     saved backward that follows it in AD then ran slower (AD 18.4
    //     against 20.0);
    //   sparse, no Hessian: 4 CTAs;
    //   sparse with the Hessian over an FP32 pool: 3 CTAs (80 registers, no
    //     spills), 19% faster than 4 (linearising forward 19.8 -> 23.5 G/s);
    //     over an FP16 pool 4 CTAs stay faster (21.5 against 19.7 G/s at 3,
    //     with the 16-byte FP16 row loads).
    if constexpr (MODE == SDFO_TRILINEAR || MODE == SDFO_TRICUBIC)
    {
        const bool hess = o.hess || o.hess6;
        // dense grids: the full 3x3 Hessian too (the bulk-copy pipeline
        // writes only the 6 unique entries)
        if (!f64 && !o.host_mapped && query_walk() && (SPARSE || !hess || o.hess))
        {
            const float* p32 = static_cast<const float*>(pts);
            // sparse 8^3 bricks: the gather specialised on the pool's storage
            constexpr bool b8 = SPARSE && BD == 8;
            const bool fp32 = v.storage == SDFO_STORAGE_FP32;
            if (!hess)
            {
                if (b8 && fp32)
                    launch_walk<MODE, SPARSE, BD, false, 4, b8 ? 1 : 0>(v, p32, n, o, s);
                else
                    launch_walk<MODE, SPARSE, BD, false, 4, b8 ? 2 : 0>(v, p32, n, o, s);
            }
            else if (fp32)
                launch_walk<MODE, SPARSE, BD, true, 3, b8 ? 1 : 0>(v, p32, n, o, s);
            else
                launch_walk<MODE, SPARSE, BD, true, 4, b8 ? 2 : 0>(v, p32, n, o, s);
            return;
        }
    }
    // The bulk-copy pipeline: dense grids, the forward that writes the
    // 6-entry Hessian (and every forward when the walk is off).  Not on sparse grids: there the
    // gathers' latency varies with the brick lookups, and the per-tile
    // barriers of a persistent CTA cost more than the prefetched points save
    // (measured: C5 forward -11%).
    if constexpr (!SPARSE && (MODE == SDFO_TRILINEAR || MODE == SDFO_TRICUBIC))
    {
        if (!f64 && launch_pipe<MODE, SPARSE, BD>(v, static_cast<const float*>(pts), n, o, s)) return;
    }
    const bool staged = !f64 && aligned16(pts) && aligned16(o.grad) && aligned16(o.unit) &&
                        aligned16(o.witness) && aligned16(o.hess6);
    if (o.hess || o.hess6)
        launch_pt2<MODE, SPARSE, BD, true>(v, pts, f64, staged, n, o, s);
    else
        launch_pt2<MODE, SPARSE, BD, false>(v, pts, f64, staged, n, o, s);
}

template <int MODE>
void launch_mode(const GridView& v, const void* pts, bool f64, int64_t n, const QueryOutputs& o,
                 cudaStream_t s)
{
    if (v.layout == SDFO_LAYOUT_DENSE)
        launch_pt<MODE, false, 0>(v, pts, f64, n, o, s);
    else if (v.bd == 8)
        launch_pt<MODE, true, 8>(v, pts, f64, n, o, s);
    else
        launch_pt<MODE, true, 0>(v, pts, f64, n, o, s);
}

template <int MODE>
void launch_bwd_mode(const GridView& v, const float* pts, int64_t n, const float* dgap,
                     const float* dgrad, float* dpts, float* dgrid, cudaStream_t s)
{
    if (query_walk() && !dgrid)
    {
        if (v.layout == SDFO_LAYOUT_DENSE)
            launch_bwd_walk<MODE, false, 0, 0>(v, pts, n, dgap, dgrad, dpts, s);
        else if (v.bd == 8 && v.storage == SDFO_STORAGE_FP32)
            launch_bwd_walk<MODE, true, 8, 1>(v, pts, n, dgap, dgrad, dpts, s);
        else if (v.bd == 8)
            launch_bwd_walk<MODE, true, 8, 2>(v, pts, n, dgap, dgrad, dpts, s);
        else
            launch_bwd_walk<MODE, true, 0, 0>(v, pts, n, dgap, dgrad, dpts, s);
        return;
    }
    const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
    if (v.layout == SDFO_LAYOUT_DENSE)
        k_query_backward<MODE, false, 0><<<blocks, kThreads, 0, s>>>(v, pts, n, dgap, dgrad, dpts, dgrid);
    else if (v.bd == 8)
        k_query_backward<MODE, true, 8><<<blocks, kThreads, 0, s>>>(v, pts, n, dgap, dgrad, dpts, dgrid);
    else
        k_query_backward<MODE, true, 0><<<blocks, kThreads, 0, s>>>(v, pts, n, dgap, dgrad, dpts, dgrid);
}

template <int MODE, bool SPARSE, int BD, bool STAGED>
void launch_saved3(const GridView& v, const SavedBackward& b, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((b.n + kThreads - 1) / kThreads);
#define SDFO_LAUNCH_SAVED(DP, DG)                                                          \
    k_backward_saved<MODE, SPARSE, BD, STAGED, DP, DG><<<blocks, kThreads, 0, s>>>(        \
        v, b.pts, b.n, b.grad, b.hess6, b.valid, b.dgap, b.dgrad, b.dpts, b.dgrid)
    if (b.dpts && b.dgrid) SDFO_LAUNCH_SAVED(true, true);
    else if (b.dpts) SDFO_LAUNCH_SAVED(true, false);
    else if (b.dgrid) SDFO_LAUNCH_SAVED(false, true);
#undef SDFO_LAUNCH_SAVED
}

template <int MODE, bool SPARSE, int BD>
void launch_saved2(const GridView& v, const SavedBackward& b, cudaStream_t s)
{
    // dL/dp alone: the bulk-copy pipeline when there is a whole tile
    if (b.dpts && !b.dgrid && launch_backward_saved_bulk(b.n, b.grad, b.hess6, b.dgap, b.dgrad, b.dpts, s))
        return;
    const bool staged = aligned16(b.pts) && aligned16(b.grad) && aligned16(b.hess6) &&
                        aligned16(b.dgrad) && aligned16(b.dpts);
    if (staged)
        launch_saved3<MODE, SPARSE, BD, true>(v, b, s);
    else
        launch_saved3<MODE, SPARSE, BD, false>(v, b, s);
}

template <int MODE>
void launch_saved_mode(const GridView& v, const SavedBackward& b, cudaStream_t s)
{
    if (v.layout == SDFO_LAYOUT_DENSE)
        launch_saved2<MODE, false, 0>(v, b, s);
    else if (v.bd == 8)
        launch_saved2<MODE, true, 8>(v, b, s);
    else
        launch_saved2<MODE, true, 0>(v, b, s);
}

} // namespace

namespace {
std::mutex g_status_mutex;
unsigned* g_status_addr[64] = {};
} // namespace

unsigned* query_pipe_status_address()
{
    int dev = 0;
    SDFO_CUDA(cudaGetDevice(&dev));
    SDFO_REQUIRE(dev >= 0 && dev < 64, SDFO_ERR_UNSUPPORTED, "device ordinal too large");
    std::lock_guard<std::mutex> lock(g_status_mutex);
    if (!g_status_addr[dev])
    {
        void* p = nullptr;
        SDFO_CUDA(cudaGetSymbolAddress(&p, g_pipe_status));
        g_status_addr[dev] = static_cast<unsigned*>(p);
    }
    return g_status_addr[dev];
}

void set_query_pipe_wait_test(unsigned limit, int withhold_first_tile)
{
    const unsigned v[2] = {limit, withhold_first_tile ? 1u : 0u};
    SDFO_CUDA(cudaMemcpyToSymbol(g_pipe_test, v, sizeof(v)));
}

unsigned query_pipe_status(bool clear)
{
    unsigned v = 0;
    SDFO_CUDA(cudaMemcpyFromSymbol(&v, g_pipe_status, sizeof(v)));
    if (clear)
    {
        const unsigned z = 0;
        SDFO_CUDA(cudaMemcpyToSymbol(g_pipe_status, &z, sizeof(z)));
    }
    return v;
}

void launch_query(const GridView& v, int mode, const void* pts, bool f64, int64_t n,
                  const QueryOutputs& o, cudaStream_t s)
{
    if (n <= 0) return;
    switch (mode)
    {
    case SDFO_FIRST_ORDER: launch_mode<SDFO_FIRST_ORDER>(v, pts, f64, n, o, s); break;
    case SDFO_SECOND_ORDER: launch_mode<SDFO_SECOND_ORDER>(v, pts, f64, n, o, s); break;
    case SDFO_TRILINEAR: launch_mode<SDFO_TRILINEAR>(v, pts, f64, n, o, s); break;
    case SDFO_TRICUBIC: launch_mode<SDFO_TRICUBIC>(v, pts, f64, n, o, s); break;
    case SDFO_CONTACT_AWARE:
        // grids without candidates answer ContactAware with Tricubic
        // (SdfOracle.cpp:187-191, 265-268, 371-374)
        if (v.ca_stride > 0)
        {
            launch_query_ca(v, pts, f64, n, o, CandidateOutputs{}, s);
            return;
        }
        launch_mode<SDFO_TRICUBIC>(v, pts, f64, n, o, s);
        break;
    default: throw Error(SDFO_ERR_INVALID_ARGUMENT, "unknown query mode");
    }
    SDFO_CHECK_LAUNCH();
}

void launch_query_backward(const GridView& v, int mode, const float* pts, int64_t n,
                           const float* dgap, const float* dgrad, float* dpts, float* dgrid,
                           cudaStream_t s)
{
    if (n <= 0) return;
    if (mode == SDFO_TRICUBIC)
        launch_bwd_mode<SDFO_TRICUBIC>(v, pts, n, dgap, dgrad, dpts, dgrid, s);
    else if (mode == SDFO_TRILINEAR)
        launch_bwd_mode<SDFO_TRILINEAR>(v, pts, n, dgap, dgrad, dpts, dgrid, s);
    else
        throw Error(SDFO_ERR_UNSUPPORTED, "query backward supports Trilinear and Tricubic");
    SDFO_CHECK_LAUNCH();
}

} // namespace sdfo

namespace sdfo {

void launch_backward_saved(const GridView& v, int mode, const SavedBackward& b, cudaStream_t s)
{
    if (b.n <= 0 || (!b.dpts && !b.dgrid)) return;
    if (mode == SDFO_TRICUBIC)
        launch_saved_mode<SDFO_TRICUBIC>(v, b, s);
    else if (mode == SDFO_TRILINEAR)
        launch_saved_mode<SDFO_TRILINEAR>(v, b, s);
    else
        throw Error(SDFO_ERR_UNSUPPORTED, "query backward supports Trilinear and Tricubic");
    SDFO_CHECK_LAUNCH();
}

} // namespace sdfo
