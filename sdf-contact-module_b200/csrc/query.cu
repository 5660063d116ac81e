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
#include "interp.cuh"

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

__device__ __forceinline__ void unit_of(const float g[3], float u[3])
{
    const float len = sqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    if (len > 1e-15f)
    {
        const float inv = 1.f / len;
        u[0] = g[0] * inv;
        u[1] = g[1] * inv;
        u[2] = g[2] * inv;
    }
    else
    {
        u[0] = 1.f;
        u[1] = 0.f;
        u[2] = 0.f;
    }
}

template <int MODE, bool SPARSE, int BD, bool HESS>
__device__ __forceinline__ bool evaluate(const GridView& g, const double p[3], Interp& r,
                                         float unit[3])
{
    const float h[3] = {(float)g.voxel[0], (float)g.voxel[1], (float)g.voxel[2]};
    if (MODE == SDFO_TRILINEAR || MODE == SDFO_TRICUBIC)
    {
        const Cell c = cell_of(g, p);
        if (!c.ok) return false;
        if (!SPARSE && MODE == SDFO_TRILINEAR && g.cell8 != nullptr)
        {
            // one 32-byte load: the 8 corner phi of the cell
            float4 a, b;
            ld256(g.cell8 + 2 * dense_index(g, c.i0, c.j0, c.k0), a, b);
            const float phi[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            r = trilinear<HESS>(phi, c.u, c.v, c.w, h);
            unit_of(r.g, unit);
            return true;
        }
        float4 cs[8];
        if (!SPARSE && MODE == SDFO_TRICUBIC && g.xpair != nullptr)
        {
            // four 32-byte loads: the x-pairs of the 4 (dj, dk) corner rows
            const int64_t base = dense_index(g, c.i0, c.j0, c.k0);
            const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const int64_t v = base + ((q & 1) ? sy : 0) + ((q & 2) ? sz : 0);
                ld256(g.xpair + 2 * v, cs[2 * q], cs[2 * q + 1]);
            }
        }
        else
        {
            int64_t idx[8];
            if (!gather_corners<SPARSE, BD>(g, c, cs, idx)) return false;
        }
        if (MODE == SDFO_TRICUBIC)
        {
            r = tricubic<HESS>(cs, c.u, c.v, c.w, h);
        }
        else
        {
            float phi[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) phi[q] = cs[q].x;
            r = trilinear<HESS>(phi, c.u, c.v, c.w, h);
        }
        unit_of(r.g, unit);
        return true;
    }
    // FirstOrder / SecondOrder at the nearest voxel (SdfOracle.cpp:448-520,
    // 600-654).
    int ijk[3];
    float dx[3];
    if (!nearest_voxel(g, p, ijk, dx)) return false;
    int64_t idx;
    if (SPARSE)
    {
        idx = sparse_index<BD>(g, ijk[0], ijk[1], ijk[2]);
        if (idx < 0) return false;
    }
    else
    {
        idx = dense_index(g, ijk[0], ijk[1], ijk[2]);
    }
    const float4 c = load_stored<BD>(g, idx);
    const float n0[3] = {c.y, c.z, c.w};
    const float first = n0[0] * dx[0] + n0[1] * dx[1] + n0[2] * dx[2];
    if (MODE == SDFO_SECOND_ORDER && g.has_hessian && g.hess6 != nullptr)
    {
        float H[6];
#pragma unroll
        for (int q = 0; q < 6; ++q) H[q] = __ldg(g.hess6 + 6 * idx + q);
        const float Hd[3] = {H[0] * dx[0] + H[1] * dx[1] + H[2] * dx[2],
                             H[1] * dx[0] + H[3] * dx[1] + H[4] * dx[2],
                             H[2] * dx[0] + H[4] * dx[1] + H[5] * dx[2]};
        r.gap = c.x + first + 0.5f * (dx[0] * Hd[0] + dx[1] * Hd[1] + dx[2] * Hd[2]);
#pragma unroll
        for (int a = 0; a < 3; ++a) r.g[a] = n0[a] + Hd[a];
#pragma unroll
        for (int q = 0; q < 6; ++q) r.H[q] = H[q];
        const float len = sqrtf(r.g[0] * r.g[0] + r.g[1] * r.g[1] + r.g[2] * r.g[2]);
        if (len > 1e-15f)
        {
#pragma unroll
            for (int a = 0; a < 3; ++a) unit[a] = r.g[a] / len;
        }
        else
        {
#pragma unroll
            for (int a = 0; a < 3; ++a) unit[a] = n0[a];
        }
        return true;
    }
    r.gap = c.x + first;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        r.g[a] = n0[a];
        unit[a] = n0[a];
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) r.H[q] = 0.f;
    return true;
}

// Block-cooperative I/O of 3-float records (points in, gradient / unit /
// witness out): the block's 256 records are one contiguous 3 KB range, moved
// with 16-byte accesses through shared memory instead of three 4-byte
// accesses per thread at a 12-byte stride.  Used when the pointers are
// 16-byte aligned (the host checks); `cnt` = records of this block.
__device__ __forceinline__ void stage_in3(float* sbuf, const float* src, int cnt)
{
    const int nf = 3 * cnt, nv = nf >> 2;
    for (int t = threadIdx.x; t < nv; t += kThreads)
        reinterpret_cast<float4*>(sbuf)[t] = __ldcs(reinterpret_cast<const float4*>(src) + t);
    for (int t = 4 * nv + threadIdx.x; t < nf; t += kThreads) sbuf[t] = __ldcs(src + t);
}

__device__ __forceinline__ void stage_out3(float* sbuf, float* dst, int cnt)
{
    const int nf = 3 * cnt, nv = nf >> 2;
    for (int t = threadIdx.x; t < nv; t += kThreads)
        __stcs(reinterpret_cast<float4*>(dst) + t, reinterpret_cast<const float4*>(sbuf)[t]);
    for (int t = 4 * nv + threadIdx.x; t < nf; t += kThreads) __stcs(dst + t, sbuf[t]);
}

template <int MODE, bool SPARSE, int BD, typename PT, bool HESS, bool STAGED>
__global__ void __launch_bounds__(kThreads) k_query(GridView g, const PT* __restrict__ pts,
                                                  int64_t n, QueryOutputs o)
{
    __shared__ __align__(16) float sbuf[STAGED ? 3 * kThreads : 1];
    const int64_t q0 = (int64_t)blockIdx.x * kThreads;
    const int64_t q = q0 + threadIdx.x;
    const bool active = q < n;
    const int cnt = (int)(n - q0 < kThreads ? n - q0 : kThreads);
    double p[3] = {0.0, 0.0, 0.0};
    if (STAGED)
    {
        stage_in3(sbuf, reinterpret_cast<const float*>(pts) + 3 * q0, cnt);
        __syncthreads();
        if (active)
        {
            p[0] = sbuf[3 * threadIdx.x];
            p[1] = sbuf[3 * threadIdx.x + 1];
            p[2] = sbuf[3 * threadIdx.x + 2];
        }
    }
    else if (active)
    {
        load_point(pts, q, p);
    }
    Interp r;
    float unit[3];
    const bool valid = active && evaluate<MODE, SPARSE, BD, HESS>(g, p, r, unit);
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
    float w[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) w[a] = valid ? (float)(p[a] - (double)r.gap * unit[a]) : 0.f;
    if (STAGED)
    {
        // o.grad / o.unit / o.witness are uniform over the block
        const float* outs[3] = {r.g, unit, w};
        float* dsts[3] = {o.grad, o.unit, o.witness};
#pragma unroll
        for (int k = 0; k < 3; ++k)
        {
            if (dsts[k] == nullptr) continue;
            __syncthreads();
            sbuf[3 * threadIdx.x] = outs[k][0];
            sbuf[3 * threadIdx.x + 1] = outs[k][1];
            sbuf[3 * threadIdx.x + 2] = outs[k][2];
            __syncthreads();
            stage_out3(sbuf, dsts[k] + 3 * q0, cnt);
        }
    }
    else if (active)
    {
        if (o.grad)
#pragma unroll
            for (int a = 0; a < 3; ++a) __stcs(o.grad + 3 * q + a, r.g[a]);
        if (o.unit)
#pragma unroll
            for (int a = 0; a < 3; ++a) __stcs(o.unit + 3 * q + a, unit[a]);
        if (o.witness)
#pragma unroll
            for (int a = 0; a < 3; ++a) __stcs(o.witness + 3 * q + a, w[a]);
    }
    if (HESS && active)
    {
        const float H9[9] = {r.H[0], r.H[1], r.H[2], r.H[1], r.H[3], r.H[4], r.H[2], r.H[4], r.H[5]};
#pragma unroll
        for (int a = 0; a < 9; ++a) __stcs(o.hess + 9 * q + a, H9[a]);
    }
}

// Backward: dL/dp = dgap * grad + H dgrad, and the scatter of dL/d(payload)
// onto the 8 corners (float4 atomics: d phi, d n).
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
    const float h[3] = {(float)g.voxel[0], (float)g.voxel[1], (float)g.voxel[2]};
    const Cell c = cell_of(g, p);
    float4 cs[8];
    int64_t idx[8];
    const bool ok = c.ok && gather_corners<SPARSE, BD>(g, c, cs, idx);
    if (!ok)
    {
        if (dpts)
        {
            dpts[3 * q + 0] = 0.f;
            dpts[3 * q + 1] = 0.f;
            dpts[3 * q + 2] = 0.f;
        }
        return;
    }
    Interp r;
    if (MODE == SDFO_TRICUBIC)
    {
        r = tricubic<true>(cs, c.u, c.v, c.w, h);
    }
    else
    {
        float phi[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) phi[k] = cs[k].x;
        r = trilinear<true>(phi, c.u, c.v, c.w, h);
    }
    if (dpts)
    {
        const float H[9] = {r.H[0], r.H[1], r.H[2], r.H[1], r.H[3], r.H[4], r.H[2], r.H[4], r.H[5]};
#pragma unroll
        for (int a = 0; a < 3; ++a)
            dpts[3 * q + a] = dG * r.g[a] + H[3 * a + 0] * dg[0] + H[3 * a + 1] * dg[1] +
                              H[3 * a + 2] * dg[2];
    }
    if (!dgrid) return;
    // Per-corner weights of gap and of grad (= d/du etc. / h).
    const float ig[3] = {dg[0] / h[0], dg[1] / h[1], dg[2] / h[2]};
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
            // d/d gx_k, gy_k, gz_k, then chain through g = n * h
            const float wgx = dG * (P1 * Q0 * R0) + ig[0] * (dP1 * Q0 * R0) +
                              ig[1] * (P1 * dQ0 * R0) + ig[2] * (P1 * Q0 * dR0);
            const float wgy = dG * (P0 * Q1 * R0) + ig[0] * (dP0 * Q1 * R0) +
                              ig[1] * (P0 * dQ1 * R0) + ig[2] * (P0 * Q1 * dR0);
            const float wgz = dG * (P0 * Q0 * R1) + ig[0] * (dP0 * Q0 * R1) +
                              ig[1] * (P0 * dQ0 * R1) + ig[2] * (P0 * Q0 * dR1);
            atomicAdd(reinterpret_cast<float4*>(dgrid) + idx[k],
                      make_float4(wphi, wgx * h[0], wgy * h[1], wgz * h[2]));
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
            atomicAdd(reinterpret_cast<float4*>(dgrid) + idx[k], make_float4(wphi, 0.f, 0.f, 0.f));
        }
    }
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

template <int MODE, bool SPARSE, int BD>
void launch_pt(const GridView& v, const void* pts, bool f64, int64_t n, const QueryOutputs& o,
               cudaStream_t s)
{
    const bool staged = !f64 && aligned16(pts) && aligned16(o.grad) && aligned16(o.unit) &&
                        aligned16(o.witness);
    if (o.hess)
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
    const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
    if (v.layout == SDFO_LAYOUT_DENSE)
        k_query_backward<MODE, false, 0><<<blocks, kThreads, 0, s>>>(v, pts, n, dgap, dgrad, dpts, dgrid);
    else if (v.bd == 8)
        k_query_backward<MODE, true, 8><<<blocks, kThreads, 0, s>>>(v, pts, n, dgap, dgrad, dpts, dgrid);
    else
        k_query_backward<MODE, true, 0><<<blocks, kThreads, 0, s>>>(v, pts, n, dgap, dgrad, dpts, dgrid);
}

} // namespace

void launch_query(const GridView& v, int mode, const void* pts, bool f64, int64_t n,
                  const QueryOutputs& o, cudaStream_t s)
{
    if (n <= 0) return;
    switch (mode)
    {
    case SDFO_FIRST_ORDER: launch_mode<SDFO_FIRST_ORDER>(v, pts, f64, n, o, s); break;
    case SDFO_SECOND_ORDER: launch_mode<SDFO_SECOND_ORDER>(v, pts, f64, n, o, s); break;
    case SDFO_TRILINEAR: launch_mode<SDFO_TRILINEAR>(v, pts, f64, n, o, s); break;
    case SDFO_TRICUBIC:
    case SDFO_CONTACT_AWARE: launch_mode<SDFO_TRICUBIC>(v, pts, f64, n, o, s); break;
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
