// Fused SDF penalty contact over quadrature points, batched over poses, with
// the forward-mode 6x6 pose Jacobian.
//
// Restates SDFContactEngine.evaluate (prototype/src/dynamics/contacts_sdf.py:
// 225-385).  Without a ContactCull every quadrature point is evaluated; with
// one, the engine's culling is applied as the reference does it: the point
// BVH's leaves overlapping the query box RA^T (bmin - rA) - m ..
// RA^T (bmax - rA) + m (m = max(narrow margin, 0.05); all points when the box
// encloses every point or no leaf overlaps it), then the narrow filter
// |Y_z| < narrow margin.  The same pass can produce measure_pair's
// ContactMeasure (contacts_sdf.py:171-214) over the BVH-kept points.  The
// force law:
//   Y = R_B^T (r_A + R_A X - r_B)                       (marker-free transform)
//   g, grad g = SDF(Y) (Trilinear or Tricubic)           (local, raw gradient)
//   active iff valid and k max(-g,0)^n > 1e-30
//   rg = R_B grad g, p = k max(-g,0)^n, fn = p rg
//   damping (c > 0, g < 0): fd = c (-(u_A - u_B).rg) rg
//   p_hat = p |grad g|, un = rg / |rg|, u_t = u - (u.un) un
//   ft = -mu p_hat u_t / sqrt(|u_t|^2 + reg^2)
//   F_A = sum w (fn + fd + ft), tau_A = sum w (x - r_A) x (fn + fd + ft)
// The Jacobian is d(F_A, tau_A)/d(dx, dtheta) for r_A += dx,
// R_A = exp([dtheta]x) R_A, propagated per point in forward mode through the
// interpolant's Hessian (no finite differences).
//
// Layout: one CTA per pose; the quadrature set (X, w) is shared by all poses
// and stays L1/L2-resident; the grid gather and interpolation are FP32; the
// per-point force law of active points, the Jacobian and the reductions
// (warp shuffles, then shared memory) are FP64.
#include <climits>

#include "interp.cuh"

namespace sdfo {
namespace {

constexpr int kContactThreads = 256;
// Jacobian pass: the points of a span of kJacSpan points that are in contact
// are listed per warp (a warp meets at most kJacSpan / 8 of them), then all
// warps share the span's list.
constexpr int kJacSpan = 4096;
constexpr int kJacPerWarp = kJacSpan / (kContactThreads / 32);

struct v3
{
    double x, y, z;
};
__device__ __forceinline__ v3 V(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator*(double s, v3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 a, v3 b)
{
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ v3 mul(const double R[9], v3 a)
{
    return {R[0] * a.x + R[1] * a.y + R[2] * a.z, R[3] * a.x + R[4] * a.y + R[5] * a.z,
            R[6] * a.x + R[7] * a.y + R[8] * a.z};
}
__device__ __forceinline__ v3 mulT(const double R[9], v3 a)
{
    return {R[0] * a.x + R[3] * a.y + R[6] * a.z, R[1] * a.x + R[4] * a.y + R[7] * a.z,
            R[2] * a.x + R[5] * a.y + R[8] * a.z};
}

template <int MODE, bool SPARSE, int BD, bool JAC>
__device__ __forceinline__ bool sample(const GridView& g, const double Y[3], float& gap, v3& grad,
                                       double Hl[6])
{
    const Cell c = cell_of(g, Y);
    if (!c.ok) return false;
    const float h[3] = {(float)g.voxel[0], (float)g.voxel[1], (float)g.voxel[2]};
    const float ih[3] = {g.ih[0], g.ih[1], g.ih[2]};
    Interp r;
    if (!SPARSE && MODE == SDFO_TRILINEAR && g.cell8 != nullptr)
    {
        float4 a, b;
        ld256(g.cell8 + 2 * dense_index(g, c.i0, c.j0, c.k0), a, b);
        const float phi[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        r = trilinear<JAC>(phi, c.u, c.v, c.w, ih);
    }
    else
    {
        float4 cs[8];
        if (!SPARSE && g.xpair != nullptr)
        {
            const int64_t base = dense_index(g, c.i0, c.j0, c.k0);
            const int64_t sy = g.nx, sz = (int64_t)g.nx * g.ny;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                ld256(g.xpair + 2 * (base + ((q & 1) ? sy : 0) + ((q & 2) ? sz : 0)), cs[2 * q],
                      cs[2 * q + 1]);
        }
        else
        {
            int64_t idx[8];
            if (!gather_corners<SPARSE, BD>(g, c, cs, idx)) return false;
        }
        if (MODE == SDFO_TRICUBIC)
        {
            r = tricubic<JAC>(cs, c.u, c.v, c.w, h, ih);
        }
        else
        {
            float phi[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) phi[q] = cs[q].x;
            r = trilinear<JAC>(phi, c.u, c.v, c.w, ih);
        }
    }
    gap = r.gap;
    grad = V(r.g[0], r.g[1], r.g[2]);
#pragma unroll
    for (int q = 0; q < 6; ++q) Hl[q] = r.H[q];
    return true;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Per-point contact state of one quadrature point at one pose.
struct PointState
{
    double p, gn, vn, udn, den, phat, dgdd, wq;
    v3 off, rg, gl, u, un, ut, fq;
    double Hl[6];
    bool damp, fric;
};

// Pose-level quantities shared by all points of a CTA.
struct PoseFrame
{
    v3 rA, rB, vA, wA, vB, wB, tl;
};

// The SDFContactEngine.evaluate force law of quadrature point i
// (contacts_sdf.py:256-385).  Returns 0 when the point is outside the grid,
// 1 when it is inside but exerts no force (k max(-g,0)^n <= 1e-30, or
// dropped by the narrow filter |Y_z| < narrow when narrow >= 0), 2 when it
// is active.  `gap` receives the gap of in-grid points; with need_gap false
// a point failing the narrow filter is not sampled (status 1, gap unset).
// HESS also records the interpolant's Hessian for the Jacobian.
template <int MODE, bool SPARSE, int BD, bool HESS>
__device__ __forceinline__ int point_state(const GridView& g, const float* __restrict__ qx,
                                           const float* __restrict__ qw, int i,
                                           const sdfo_body_state& sA, const sdfo_body_state& sB,
                                           const PoseFrame& f, const sdfo_contact_params& prm,
                                           double narrow, bool need_gap, PointState& st,
                                           double& gap_out)
{
    const v3 X = V(__ldg(qx + 3 * i), __ldg(qx + 3 * i + 1), __ldg(qx + 3 * i + 2));
    st.off = mul(sA.R, X);                   // x_w - r_A
    const v3 Yv = mulT(sB.R, st.off) + f.tl; // body-B local point
    const bool narrow_ok = !(narrow >= 0.0) || fabs(Yv.z) < narrow;
    if (!narrow_ok && !need_gap) return 1;
    const double Y[3] = {Yv.x, Yv.y, Yv.z};
    float gapf;
    if (!sample<MODE, SPARSE, BD, HESS>(g, Y, gapf, st.gl, st.Hl)) return 0;
    const double gap = gapf;
    gap_out = gap;
    if (!narrow_ok) return 1;
    const double delta = gap < 0.0 ? -gap : 0.0;
    const double dpow = prm.order == 2.0 ? delta * delta : prm.order == 1.0 ? delta : pow(delta, prm.order);
    st.p = prm.stiffness * dpow;
    if (!(st.p > 1e-30)) return 1;
    st.wq = (double)__ldg(qw + i);
    const v3 xw = f.rA + st.off;
    st.rg = mul(sB.R, st.gl);
    st.gn = sqrt(dot(st.gl, st.gl));
    st.fq = st.p * st.rg;
    const v3 uA = f.vA + cross(f.wA, st.off);
    const v3 uB = f.vB + cross(f.wB, xw - f.rB);
    st.u = uA - uB;
    st.damp = prm.damping > 0.0 && gap < 0.0;
    st.vn = dot(st.u, st.rg);
    if (st.damp) st.fq = st.fq + (prm.damping * (-st.vn)) * st.rg;
    const double gsafe = st.gn > 1e-30 ? st.gn : 1e-30;
    st.un = (1.0 / gsafe) * st.rg;
    st.udn = dot(st.u, st.un);
    st.ut = st.u - st.udn * st.un;
    st.den = sqrt(dot(st.ut, st.ut) + prm.regularizer * prm.regularizer);
    st.phat = st.p * st.gn;
    st.fric = prm.friction * st.phat > 0.0;
    if (st.fric) st.fq = st.fq + (-prm.friction * st.phat / st.den) * st.ut;
    st.dgdd = -prm.stiffness * (prm.order == 2.0 ? 2.0 * delta
                                : prm.order == 1.0 ? 1.0
                                                   : prm.order * pow(delta, prm.order - 1.0));
    return 2;
}

// Column j of the point's d(f, x f)/d(dx, dtheta), weighted by w.
__device__ __forceinline__ void jacobian_column(const PointState& st, const sdfo_body_state& sB,
                                                const PoseFrame& f, const sdfo_contact_params& prm,
                                                int j, double col[6])
{
    const double Hm[9] = {st.Hl[0], st.Hl[1], st.Hl[2], st.Hl[1], st.Hl[3],
                          st.Hl[4], st.Hl[2], st.Hl[4], st.Hl[5]};
    v3 dxw, doff;
    if (j < 3)
    {
        dxw = V(j == 0, j == 1, j == 2);
        doff = V(0.0, 0.0, 0.0);
    }
    else
    {
        doff = cross(V(j == 3, j == 4, j == 5), st.off);
        dxw = doff;
    }
    const v3 dYl = mulT(sB.R, dxw);
    const v3 dgl = V(Hm[0] * dYl.x + Hm[1] * dYl.y + Hm[2] * dYl.z,
                     Hm[3] * dYl.x + Hm[4] * dYl.y + Hm[5] * dYl.z,
                     Hm[6] * dYl.x + Hm[7] * dYl.y + Hm[8] * dYl.z);
    const double dg = dot(st.gl, dYl);
    const v3 drg = mul(sB.R, dgl);
    const double dp = st.dgdd * dg; // p = k delta^n, delta = -g
    v3 dfq = dp * st.rg + st.p * drg;
    const v3 du = cross(f.wA, doff) - cross(f.wB, dxw);
    if (st.damp)
    {
        const double dvn = dot(du, st.rg) + dot(st.u, drg);
        dfq = dfq + (-prm.damping) * (dvn * st.rg + st.vn * drg);
    }
    if (st.fric)
    {
        const double gsafe = st.gn > 1e-30 ? st.gn : 1e-30;
        const double dgn = st.gn > 1e-30 ? dot(st.gl, dgl) / st.gn : 0.0;
        const double dphat = dp * st.gn + st.p * dgn;
        const v3 dun = (1.0 / gsafe) * (st.gn > 1e-30 ? drg - dot(st.un, drg) * st.un : drg);
        const double dudn = dot(du, st.un) + dot(st.u, dun);
        const v3 dut = du - dudn * st.un - st.udn * dun;
        const double dden = dot(st.ut, dut) / st.den;
        dfq = dfq + (-prm.friction) * ((dphat / st.den) * st.ut + (st.phat / st.den) * dut -
                                       (st.phat * dden / (st.den * st.den)) * st.ut);
    }
    const v3 dtq = cross(doff, st.fq) + cross(st.off, dfq);
    col[0] = st.wq * dfq.x;
    col[1] = st.wq * dfq.y;
    col[2] = st.wq * dfq.z;
    col[3] = st.wq * dtq.x;
    col[4] = st.wq * dtq.y;
    col[5] = st.wq * dtq.z;
}

// One CTA per pose.  Per chunk of 256 quadrature points: every thread
// evaluates its point (no Hessian) and accumulates F, tau; with JAC the
// chunk's active points (typically a small fraction) are then compacted in
// point order into the first threads, which re-evaluate them with the
// interpolant's Hessian and form the six Jacobian columns -- so only
// ceil(active / 32) warps run the FP64 derivative code, with full lanes.
// Resident CTAs per SM asked of the register allocator (256 threads each).
#ifndef SDFO_CONTACT_MIN_BLOCKS
#define SDFO_CONTACT_MIN_BLOCKS 3
#endif
#ifndef SDFO_CONTACT_JAC_MIN_BLOCKS
#define SDFO_CONTACT_JAC_MIN_BLOCKS 2
#endif

// Lexicographic (gap, key) minimum for measure_pair's argmin: the reference
// takes the first minimum in its point order, `key` is the point's position
// in that order.
struct MinRec
{
    double gap;
    int key;
    int i;
};

__device__ __forceinline__ bool less_rec(const MinRec& a, const MinRec& b)
{
    return a.gap < b.gap || (a.gap == b.gap && a.key < b.key);
}

__device__ __forceinline__ MinRec warp_min(MinRec r)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        MinRec q;
        q.gap = __shfl_down_sync(0xffffffffu, r.gap, o);
        q.key = __shfl_down_sync(0xffffffffu, r.key, o);
        q.i = __shfl_down_sync(0xffffffffu, r.i, o);
        if (less_rec(q, r)) r = q;
    }
    return r;
}

__device__ __forceinline__ int warp_isum(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// EXT: the culled / measuring variant (ContactCull, measures); without it
// every point is evaluated and no measure is produced.
template <int MODE, bool SPARSE, int BD, bool JAC, bool EXT>
__global__ void __launch_bounds__(kContactThreads,
                                  JAC ? SDFO_CONTACT_JAC_MIN_BLOCKS : SDFO_CONTACT_MIN_BLOCKS)
    k_contact(GridView g, const float* __restrict__ qx, const float* __restrict__ qw, int nq,
              const sdfo_body_state* __restrict__ poses, const sdfo_body_state* __restrict__ body_b,
              sdfo_contact_params prm, double* __restrict__ ft, double* __restrict__ jac, ContactCull cull,
              sdfo_contact_measure* __restrict__ meas)
{
    constexpr int kWarps = kContactThreads / 32;
    const int pose = blockIdx.x;
    __shared__ sdfo_body_state sA, sB;
    __shared__ double red[kWarps][6];
    __shared__ double sjac[JAC ? kWarps : 1][JAC ? 36 : 1];
    __shared__ int s_list[JAC ? kJacSpan : 1];
    __shared__ int s_wcnt[kWarps];
    __shared__ unsigned s_mask[EXT ? kMaxCullLeaves / 32 : 1];
    __shared__ double s_box[6];
    __shared__ int s_full;
    __shared__ MinRec s_min[EXT ? kWarps : 1];
    __shared__ int s_cnt[EXT ? kWarps : 1][2];
    __shared__ int s_prefix;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0)
    {
        sA = poses[pose];
        sB = *body_b;
    }
    if (JAC)
        for (int t = lane; t < 36; t += 32) sjac[warp][t] = 0.0;
    __syncthreads();
    PoseFrame f;
    f.rA = V(sA.r[0], sA.r[1], sA.r[2]);
    f.rB = V(sB.r[0], sB.r[1], sB.r[2]);
    f.vA = V(sA.v[0], sA.v[1], sA.v[2]);
    f.wA = V(sA.w[0], sA.w[1], sA.w[2]);
    f.vB = V(sB.v[0], sB.v[1], sB.v[2]);
    f.wB = V(sB.w[0], sB.w[1], sB.w[2]);
    f.tl = mulT(sB.R, f.rA - f.rB); // R_B^T (r_A - r_B)

    // broad phase: AABB_BVH.query(bmin_local, bmax_local) (bvh.py:62-80)
    bool full = true;
    if (EXT && cull.enabled)
    {
        if (threadIdx.x == 0)
        {
            const v3 lo = mulT(sA.R, V(cull.bmin[0], cull.bmin[1], cull.bmin[2]) - f.rA);
            const v3 hi = mulT(sA.R, V(cull.bmax[0], cull.bmax[1], cull.bmax[2]) - f.rA);
            s_box[0] = lo.x - cull.box_margin;
            s_box[1] = lo.y - cull.box_margin;
            s_box[2] = lo.z - cull.box_margin;
            s_box[3] = hi.x + cull.box_margin;
            s_box[4] = hi.y + cull.box_margin;
            s_box[5] = hi.z + cull.box_margin;
            bool enc = true;
            for (int a = 0; a < 3; ++a)
                enc = enc && s_box[a] <= cull.root[a] && s_box[3 + a] >= cull.root[3 + a];
            s_full = enc ? 1 : 0;
        }
        for (int w = threadIdx.x; w < (cull.nleaves + 31) / 32; w += kContactThreads) s_mask[w] = 0u;
        __syncthreads();
        full = s_full != 0;
        if (!full)
        {
            bool any = false;
            for (int l = threadIdx.x; l < cull.nleaves; l += kContactThreads)
            {
                const double* b = cull.leaf_box + 6 * (int64_t)l;
                const bool skip = b[3] < s_box[0] || b[4] < s_box[1] || b[5] < s_box[2] || b[0] > s_box[3] ||
                                  b[1] > s_box[4] || b[2] > s_box[5];
                if (!skip)
                {
                    atomicOr(&s_mask[l >> 5], 1u << (l & 31));
                    any = true;
                }
            }
            full = __syncthreads_or(any) == 0; // no leaf: every point (contacts_sdf.py:268-269)
        }
    }
    const double narrow = EXT && cull.enabled ? cull.narrow_margin : -1.0;
    const bool want_force = ft != nullptr;
    const bool want_meas = EXT && meas != nullptr;
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    MinRec best{INFINITY, INT_MAX, -1};
    int nvalid = 0, nactive = 0;

    // Spans of kJacSpan points (one span over all points without the
    // Jacobian).  First every point's forward; with the Jacobian, each warp
    // lists its points in contact, in point order, with no barrier.  Then
    // the span's list is shared out: group k of 32 consecutive entries to
    // warp k mod 8, so all warps carry the FP64 Jacobian work, and the sums
    // run in a fixed order (repeated runs are bit-identical).  Block-uniform
    // trip counts: the barriers and warp reductions below see every thread.
    for (int s0 = 0; s0 < nq; s0 += JAC ? kJacSpan : nq)
    {
    const int s1 = JAC ? min(nq, s0 + kJacSpan) : nq;
    int wcnt = 0; // this warp's listed points in the span (warp-uniform)
    for (int i0 = s0; i0 < s1; i0 += kContactThreads)
    {
        const int i = i0 + threadIdx.x;
        bool act = false;
        if (i < s1)
        {
            bool sel = true;
            if (EXT && !full)
            {
                const int l = __ldg(cull.pleaf + i);
                sel = (s_mask[l >> 5] >> (l & 31)) & 1u;
            }
            if (sel)
            {
                PointState st;
                double gap = 0.0;
                const int status =
                    point_state<MODE, SPARSE, BD, false>(g, qx, qw, i, sA, sB, f, prm, narrow, want_meas, st, gap);
                if (want_meas && status > 0)
                {
                    ++nvalid;
                    if (gap < 0.0) ++nactive;
                    const MinRec r{gap, full ? (cull.porig ? __ldg(cull.porig + i) : i) : i, i};
                    if (less_rec(r, best)) best = r;
                }
                act = status == 2 && want_force;
                if (act)
                {
                    const v3 tq = cross(st.off, st.fq);
                    acc[0] += st.wq * st.fq.x;
                    acc[1] += st.wq * st.fq.y;
                    acc[2] += st.wq * st.fq.z;
                    acc[3] += st.wq * tq.x;
                    acc[4] += st.wq * tq.y;
                    acc[5] += st.wq * tq.z;
                }
            }
        }
        if (JAC)
        {
            const unsigned m = __ballot_sync(0xffffffffu, act);
            if (act) s_list[warp * kJacPerWarp + wcnt + __popc(m & ((1u << lane) - 1u))] = i;
            wcnt += __popc(m);
        }
    }
    if (JAC)
    {
        if (lane == 0) s_wcnt[warp] = wcnt;
        __syncthreads();
        int total = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) total += s_wcnt[w];
        for (int k = warp; 32 * k < total; k += kWarps) // warp-uniform
        {
            const int e = 32 * k + lane;
            bool mine = e < total;
            int idx = 0;
            if (mine)
            {
                // entry e of the span's list: warp src's list, position rem
                int rem = e, src = 0;
#pragma unroll
                for (int w = 0; w < kWarps; ++w)
                {
                    const int c = s_wcnt[w];
                    if (src == w && rem >= c)
                    {
                        rem -= c;
                        ++src;
                    }
                }
                idx = s_list[src * kJacPerWarp + rem];
            }
            PointState st;
            double gap = 0.0;
            mine = mine && point_state<MODE, SPARSE, BD, true>(g, qx, qw, idx, sA, sB, f, prm, narrow, false,
                                                               st, gap) == 2;
#pragma unroll 1
            for (int j = 0; j < 6; ++j)
            {
                double col[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                if (mine) jacobian_column(st, sB, f, prm, j, col);
#pragma unroll
                for (int r = 0; r < 6; ++r)
                {
                    const double sum = warp_sum(col[r]);
                    if (lane == 0) sjac[warp][6 * r + j] += sum;
                }
            }
        }
        __syncthreads(); // s_list and s_wcnt are rewritten by the next span
    }
    }
    if (want_force)
    {
#pragma unroll
        for (int q = 0; q < 6; ++q)
        {
            const double s = warp_sum(acc[q]);
            if (lane == 0) red[warp][q] = s;
        }
    }
    if (want_meas)
    {
        const MinRec r = warp_min(best);
        const int nv = warp_isum(nvalid), na = warp_isum(nactive);
        if (lane == 0)
        {
            s_min[warp] = r;
            s_cnt[warp][0] = nv;
            s_cnt[warp][1] = na;
        }
        if (threadIdx.x == 0) s_prefix = 0;
    }
    __syncthreads();
    if (want_force && threadIdx.x < 6)
    {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += red[w][threadIdx.x];
        ft[6 * (int64_t)pose + threadIdx.x] = s;
    }
    if (JAC && jac != nullptr && threadIdx.x < 36)
    {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) s += sjac[w][threadIdx.x];
        jac[36 * (int64_t)pose + threadIdx.x] = s;
    }
    if (!want_meas) return;
    MinRec b = s_min[0];
    int nv = s_cnt[0][0], na = s_cnt[0][1];
#pragma unroll
    for (int w = 1; w < kWarps; ++w)
    {
        if (less_rec(s_min[w], b)) b = s_min[w];
        nv += s_cnt[w][0];
        na += s_cnt[w][1];
    }
    // position of the minimum in the broad phase's point list: the points of
    // the kept leaves before its own
    if (nv > 0 && !full)
    {
        const int lb = __ldg(cull.pleaf + b.i);
        int part = 0;
        for (int l = threadIdx.x; l < lb; l += kContactThreads)
            if ((s_mask[l >> 5] >> (l & 31)) & 1u) part += __ldg(cull.leaf_start + l + 1) - __ldg(cull.leaf_start + l);
        part = warp_isum(part);
        if (lane == 0 && part) atomicAdd(&s_prefix, part);
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    sdfo_contact_measure out;
    out.reserved0 = 0;
    out.active_count = na;
    out.valid_count = nv;
    if (nv == 0)
    {
        out.gap = INFINITY;
        out.penetration = 0.0;
        out.normal_velocity = 0.0;
        out.min_point_index = -1;
    }
    else
    {
        out.gap = b.gap;
        out.penetration = b.gap < 0.0 ? -b.gap : 0.0;
        out.min_point_index = full ? b.key : s_prefix + (b.i - __ldg(cull.leaf_start + __ldg(cull.pleaf + b.i)));
        // normal relative velocity at the minimum (contacts_sdf.py:199-211)
        const v3 X = V(__ldg(qx + 3 * b.i), __ldg(qx + 3 * b.i + 1), __ldg(qx + 3 * b.i + 2));
        const v3 off = mul(sA.R, X);
        const v3 Yv = mulT(sB.R, off) + f.tl;
        const double Y[3] = {Yv.x, Yv.y, Yv.z};
        float gapf;
        v3 gl;
        double Hl[6];
        sample<MODE, SPARSE, BD, false>(g, Y, gapf, gl, Hl);
        const double gn = sqrt(dot(gl, gl));
        const v3 un = gn > 1e-30 ? (1.0 / gn) * gl : V(0.0, 0.0, 1.0);
        v3 nw = mul(sB.R, un);
        const double nn = sqrt(dot(nw, nw));
        if (nn > 1e-30) nw = (1.0 / nn) * nw;
        const v3 xw = f.rA + off;
        const v3 uA = f.vA + cross(f.wA, off);
        const v3 uB = f.vB + cross(f.wB, xw - f.rB);
        out.normal_velocity = dot(uA - uB, nw);
    }
    meas[pose] = out;
}

struct ContactLaunch
{
    const float* qx;
    const float* qw;
    int nq;
    const sdfo_body_state* pa;
    int np;
    const sdfo_body_state* pb;
    sdfo_contact_params prm;
    double* ft;
    double* jac;
    ContactCull cull;
    sdfo_contact_measure* meas;
};

template <int MODE, bool SPARSE, int BD, bool EXT>
void launch4(const GridView& v, const ContactLaunch& c, cudaStream_t s)
{
    if (c.jac)
        k_contact<MODE, SPARSE, BD, true, EXT><<<c.np, kContactThreads, 0, s>>>(v, c.qx, c.qw, c.nq, c.pa, c.pb,
                                                                                c.prm, c.ft, c.jac, c.cull, c.meas);
    else
        k_contact<MODE, SPARSE, BD, false, EXT><<<c.np, kContactThreads, 0, s>>>(v, c.qx, c.qw, c.nq, c.pa, c.pb,
                                                                                 c.prm, c.ft, c.jac, c.cull, c.meas);
}

template <int MODE, bool SPARSE, int BD>
void launch3(const GridView& v, const ContactLaunch& c, cudaStream_t s)
{
    if (c.cull.enabled || c.meas)
        launch4<MODE, SPARSE, BD, true>(v, c, s);
    else
        launch4<MODE, SPARSE, BD, false>(v, c, s);
}

template <int MODE>
void launch2(const GridView& v, const ContactLaunch& c, cudaStream_t s)
{
    if (v.layout == SDFO_LAYOUT_DENSE)
        launch3<MODE, false, 0>(v, c, s);
    else if (v.bd == 8)
        launch3<MODE, true, 8>(v, c, s);
    else
        launch3<MODE, true, 0>(v, c, s);
}

} // namespace

void launch_contact(const GridView& v, int mode, const float* qx, const float* qw, int64_t nq,
                    const sdfo_body_state* pose_a, int64_t np, const sdfo_body_state* body_b,
                    const sdfo_contact_params& prm, double* ft, double* jac, cudaStream_t s,
                    const ContactCull* cull, sdfo_contact_measure* meas)
{
    if (np <= 0) return;
    ContactLaunch c{qx, qw, (int)nq, pose_a, (int)np, body_b, prm, ft, jac, ContactCull{}, meas};
    if (cull) c.cull = *cull;
    if (mode == SDFO_TRICUBIC)
        launch2<SDFO_TRICUBIC>(v, c, s);
    else
        launch2<SDFO_TRILINEAR>(v, c, s);
    SDFO_CHECK_LAUNCH();
}

} // namespace sdfo
