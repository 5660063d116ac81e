// Fused SDF penalty contact over quadrature points, batched over poses, with
// the forward-mode 6x6 pose Jacobian.
//
// Restates SDFContactEngine.evaluate (prototype/src/dynamics/contacts_sdf.py:
// 225-385) without its culling heuristics (AABB broad phase, point BVH, the
// |Y_z| < margin narrow filter), which only skip points that contribute no
// force:
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
#include "interp.cuh"

namespace sdfo {
namespace {

constexpr int kContactThreads = 256;

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
    float4 cs[8];
    int64_t idx[8];
    if (!gather_corners<SPARSE, BD>(g, c, cs, idx)) return false;
    const float h[3] = {(float)g.voxel[0], (float)g.voxel[1], (float)g.voxel[2]};
    Interp r;
    if (MODE == SDFO_TRICUBIC)
    {
        r = tricubic<JAC>(cs, c.u, c.v, c.w, h);
    }
    else
    {
        float phi[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) phi[q] = cs[q].x;
        r = trilinear<JAC>(phi, c.u, c.v, c.w, h);
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

template <int MODE, bool SPARSE, int BD, bool JAC>
__global__ void __launch_bounds__(kContactThreads)
    k_contact(GridView g, const float* __restrict__ qx, const float* __restrict__ qw, int nq,
              const sdfo_body_state* __restrict__ poses, const sdfo_body_state* __restrict__ body_b,
              sdfo_contact_params prm, double* __restrict__ ft, double* __restrict__ jac)
{
    constexpr int NACC = JAC ? 42 : 6;
    const int pose = blockIdx.x;
    __shared__ sdfo_body_state sA, sB;
    __shared__ double red[kContactThreads / 32][NACC];
    if (threadIdx.x == 0)
    {
        sA = poses[pose];
        sB = *body_b;
    }
    __syncthreads();
    const v3 rA = V(sA.r[0], sA.r[1], sA.r[2]), rB = V(sB.r[0], sB.r[1], sB.r[2]);
    const v3 vA = V(sA.v[0], sA.v[1], sA.v[2]), wA = V(sA.w[0], sA.w[1], sA.w[2]);
    const v3 vB = V(sB.v[0], sB.v[1], sB.v[2]), wB = V(sB.w[0], sB.w[1], sB.w[2]);
    const v3 tl = mulT(sB.R, rA - rB); // R_B^T (r_A - r_B)
    double acc[NACC];
#pragma unroll
    for (int q = 0; q < NACC; ++q) acc[q] = 0.0;

    for (int i = threadIdx.x; i < nq; i += kContactThreads)
    {
        const v3 X = V(__ldg(qx + 3 * i), __ldg(qx + 3 * i + 1), __ldg(qx + 3 * i + 2));
        const v3 off = mul(sA.R, X);           // x_w - r_A
        const v3 Yv = mulT(sB.R, off) + tl;    // body-B local point
        const double Y[3] = {Yv.x, Yv.y, Yv.z};
        float gapf;
        v3 gl;
        double Hl[6];
        if (!sample<MODE, SPARSE, BD, JAC>(g, Y, gapf, gl, Hl)) continue;
        const double gap = gapf;
        const double delta = gap < 0.0 ? -gap : 0.0;
        const double dpow = prm.order == 2.0 ? delta * delta
                          : prm.order == 1.0 ? delta
                                             : pow(delta, prm.order);
        const double p = prm.stiffness * dpow;
        if (!(p > 1e-30)) continue;
        const double wq = (double)__ldg(qw + i);
        const v3 xw = rA + off;
        const v3 rg = mul(sB.R, gl);
        const double gn = sqrt(dot(gl, gl));
        v3 fq = p * rg;
        const v3 uA = vA + cross(wA, off);
        const v3 offB = xw - rB;
        const v3 uB = vB + cross(wB, offB);
        const v3 u = uA - uB;
        const bool damp = prm.damping > 0.0 && gap < 0.0;
        const double vn = dot(u, rg);
        if (damp) fq = fq + (prm.damping * (-vn)) * rg;
        const double gsafe = gn > 1e-30 ? gn : 1e-30;
        const v3 un = (1.0 / gsafe) * rg;
        const double udn = dot(u, un);
        const v3 ut = u - udn * un;
        const double utn2 = dot(ut, ut);
        const double den = sqrt(utn2 + prm.regularizer * prm.regularizer);
        const double phat = p * gn;
        const bool fric = prm.friction * phat > 0.0;
        if (fric) fq = fq + (-prm.friction * phat / den) * ut;
        const v3 tq = cross(off, fq);
        acc[0] += wq * fq.x;
        acc[1] += wq * fq.y;
        acc[2] += wq * fq.z;
        acc[3] += wq * tq.x;
        acc[4] += wq * tq.y;
        acc[5] += wq * tq.z;
        if (JAC)
        {
            // world Hessian of g: H_w = R_B H_l R_B^T
            const double Hm[9] = {Hl[0], Hl[1], Hl[2], Hl[1], Hl[3], Hl[4], Hl[2], Hl[4], Hl[5]};
            const double dgdd = -prm.stiffness *
                                (prm.order == 2.0 ? 2.0 * delta
                                 : prm.order == 1.0 ? 1.0
                                                    : prm.order * pow(delta, prm.order - 1.0));
#pragma unroll 1
            for (int j = 0; j < 6; ++j)
            {
                // dx_w and d(off) for parameter j
                v3 dxw, doff;
                if (j < 3)
                {
                    dxw = V(j == 0, j == 1, j == 2);
                    doff = V(0.0, 0.0, 0.0);
                }
                else
                {
                    const v3 e = V(j == 3, j == 4, j == 5);
                    doff = cross(e, off);
                    dxw = doff;
                }
                const v3 dYl = mulT(sB.R, dxw);
                const v3 dgl = V(Hm[0] * dYl.x + Hm[1] * dYl.y + Hm[2] * dYl.z,
                                 Hm[3] * dYl.x + Hm[4] * dYl.y + Hm[5] * dYl.z,
                                 Hm[6] * dYl.x + Hm[7] * dYl.y + Hm[8] * dYl.z);
                const double dg = dot(gl, dYl);
                const v3 drg = mul(sB.R, dgl);
                const double dp = dgdd * dg; // p = k delta^n, delta = -g
                v3 dfq = dp * rg + p * drg;
                const v3 duA = cross(wA, doff);
                const v3 duB = cross(wB, dxw);
                const v3 du = duA - duB;
                if (damp)
                {
                    const double dvn = dot(du, rg) + dot(u, drg);
                    dfq = dfq + (-prm.damping) * (dvn * rg + vn * drg);
                }
                if (fric)
                {
                    const double dgn = gn > 1e-30 ? dot(gl, dgl) / gn : 0.0;
                    const double dphat = dp * gn + p * dgn;
                    const v3 dun = gn > 1e-30 ? (1.0 / gn) * (drg - dot(un, drg) * un)
                                              : (1.0 / gsafe) * drg;
                    const double dudn = dot(du, un) + dot(u, dun);
                    const v3 dut = du - dudn * un - udn * dun;
                    const double dden = dot(ut, dut) / den;
                    dfq = dfq + (-prm.friction) * ((dphat / den) * ut + (phat / den) * dut -
                                                   (phat * dden / (den * den)) * ut);
                }
                const v3 dtq = cross(doff, fq) + cross(off, dfq);
                acc[6 + 0 * 6 + j] += wq * dfq.x;
                acc[6 + 1 * 6 + j] += wq * dfq.y;
                acc[6 + 2 * 6 + j] += wq * dfq.z;
                acc[6 + 3 * 6 + j] += wq * dtq.x;
                acc[6 + 4 * 6 + j] += wq * dtq.y;
                acc[6 + 5 * 6 + j] += wq * dtq.z;
            }
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < NACC; ++q)
    {
        const double s = warp_sum(acc[q]);
        if (lane == 0) red[warp][q] = s;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < NACC; q += kContactThreads)
    {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kContactThreads / 32; ++w) s += red[w][q];
        if (q < 6)
            ft[6 * (int64_t)pose + q] = s;
        else if (jac)
            jac[36 * (int64_t)pose + (q - 6)] = s;
    }
}

template <int MODE, bool SPARSE, int BD>
void launch3(const GridView& v, const float* qx, const float* qw, int nq, const sdfo_body_state* pa,
             int np, const sdfo_body_state* pb, const sdfo_contact_params& prm, double* ft,
             double* jac, cudaStream_t s)
{
    if (jac)
        k_contact<MODE, SPARSE, BD, true><<<np, kContactThreads, 0, s>>>(v, qx, qw, nq, pa, pb, prm, ft, jac);
    else
        k_contact<MODE, SPARSE, BD, false><<<np, kContactThreads, 0, s>>>(v, qx, qw, nq, pa, pb, prm, ft, jac);
}

template <int MODE>
void launch2(const GridView& v, const float* qx, const float* qw, int nq, const sdfo_body_state* pa,
             int np, const sdfo_body_state* pb, const sdfo_contact_params& prm, double* ft,
             double* jac, cudaStream_t s)
{
    if (v.layout == SDFO_LAYOUT_DENSE)
        launch3<MODE, false, 0>(v, qx, qw, nq, pa, np, pb, prm, ft, jac, s);
    else if (v.bd == 8)
        launch3<MODE, true, 8>(v, qx, qw, nq, pa, np, pb, prm, ft, jac, s);
    else
        launch3<MODE, true, 0>(v, qx, qw, nq, pa, np, pb, prm, ft, jac, s);
}

} // namespace

void launch_contact(const GridView& v, int mode, const float* qx, const float* qw, int64_t nq,
                    const sdfo_body_state* pose_a, int64_t np, const sdfo_body_state* body_b,
                    const sdfo_contact_params& prm, double* ft, double* jac, cudaStream_t s)
{
    if (np <= 0) return;
    if (mode == SDFO_TRICUBIC)
        launch2<SDFO_TRICUBIC>(v, qx, qw, (int)nq, pose_a, (int)np, body_b, prm, ft, jac, s);
    else
        launch2<SDFO_TRILINEAR>(v, qx, qw, (int)nq, pose_a, (int)np, body_b, prm, ft, jac, s);
    SDFO_CHECK_LAUNCH();
}

} // namespace sdfo
