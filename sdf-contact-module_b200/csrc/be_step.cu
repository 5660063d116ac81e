// Backward-Euler contact steps on the GPU: BackwardEulerIntegrator.step
// (prototype/src/integrators/implicit_be.py:131-181) for batches of
// independent scenes.  Each scene is one free rigid body A carrying the
// quadrature set of a contact pair, against the fixed body B whose dense grid
// the pair is bound to (one movable body, one contact pair, no joints or
// drives).  One CTA runs one scene's whole adaptive step:
//   * measure_pair of the start state; a region found penetrating becomes
//     IMPACTING (_activate_initially_penetrating_regions, :223-233);
//   * h_cap = min(dt, the region's dt_current when active, else dt_normal);
//   * for an inactive region, a trial BE step over h_cap without contact
//     forces and, when it crosses into contact, the bisection of
//     _bisect_toi_pair (:336-394) with a BE trial step per halving;
//   * the real BE step (to the TOI, or over h_cap with contact forces when
//     the region is active) and the phase state machine
//     (_refresh_contact_states, :248-295).
// A BE step (_step_be, :468-505) is Newton on V = (v, w): residual
// M (V - V0)/h + C - Q (:536-604), the reference's diagonal tangent
// (_contact_tangent / _tangent, :606-687), exact solve of its two blocks,
// backtracking line search over 1, 1/2, .. 1/16 (:689-697).  Contact forces
// follow SDFContactEngine.evaluate with its culling and linearisation cache
// (contacts_sdf.py:225-385): the first evaluation of a step queries the
// narrow-filtered points and stores (g, grad, valid) by position together
// with the SDF-frame translation; later evaluations with the same number of
// narrow-filtered points use g + grad . (t - t_ref).
//
// Tangent modes (sdfo_be_params.tangent):
//   * SDFO_BE_TANGENT_REFERENCE: the reference's method as above -- the
//     linearisation cache inside a step and the heuristic diagonal tangent;
//   * SDFO_BE_TANGENT_EXACT: every residual evaluates contact exactly (no
//     cache) and Newton uses the analytic dR/dV: M/h, the derivatives of the
//     rotational inertia and gyroscopic terms through R(w), and the contact
//     block Jv + Jp diag(h I, h J_l(h w)), where Jp = d(F, tau)/d(dx, dtheta)
//     (R <- exp([dtheta]x) R) at fixed velocities and Jv = d(F, tau)/d(v, w)
//     at a fixed pose come from the force law differentiated per point with
//     the trilinear Hessian, reduced in FP64 in a fixed order (warp shuffles,
//     then warps in order), and the 6x6 system is solved by Gaussian
//     elimination with partial pivoting.  Each mode is its own kernel
//     instantiation, so the reference mode keeps its register budget.
//
// Grid samples are FP64 trilinear on the grid's FP64 values, written as the
// prototype's TrilinearSDFGrid.query_batch (prototype/src/sdf_grid.py:
// 138-204); this translation unit is compiled with -fmad=false so that every
// FP64 expression is evaluated in source order, as NumPy does.
//
// Control flow: every thread runs the same loops and branches; decisions and
// all scalar state live in shared memory, written by thread 0 between
// barriers; the contact passes use all threads.
#include <cfloat>
#include <climits>
#include <cstring>

#include "sdfo_internal.cuh"

namespace sdfo {
namespace {

// Threads per scene: 256 (one CTA per scene, two scenes per SM), 128 (four
// per SM) or 32 (one warp per scene, eight scenes per CTA, sixteen per SM:
// warp-level synchronisation instead of CTA barriers).
constexpr int kMaxT = 256;
constexpr int kMaxWarps = kMaxT / 32;

enum : int
{
    kInactive = 0,
    kImpacting = 2,
    kActive = 3,
    kStable = 4,
    kLeaving = 5
};

struct Body
{
    double r[3], R[9], v[3], w[3], t;
};

struct BeView
{
    GridView g;
    const double* phi64;
    int nq, nleaves, cull;
    const double* px;         // stored (leaf) order
    const double* pw;
    const int32_t* pleaf;
    const double* ox;         // original order
    const double* ow;
    const double* leaf_box;
    double root[6], bmin[3], bmax[3], box_margin, narrow;
    double rB[3], RB[9], vB[3], wB[3];
    double mass, Ib[9], gravity[3], area;
    sdfo_contact_params c;
    sdfo_be_params p;
    double* cg;               // cache scratch, nq per scene
    double* cgrad;            // 3 nq per scene
    unsigned char* cvalid;    // nq per scene
    unsigned long long* stats; // Newton iterations, residual evaluations, BE solves
};

constexpr int kJac = 72; // Jp (36) then Jv (36), row-major 6x6 each
// Cache positions without per-chunk barriers (CTA per scene): one count per
// (chunk, warp) of the narrow-filtered points, then their exclusive prefix;
// up to kPrefCap entries (32,768 points at 256 threads), larger point sets
// take the per-chunk block scan.
constexpr int kPrefCap = 1024;

struct MinRec
{
    double gap;
    int key; // position in the kept list
    int i;   // index into the point arrays
};

struct Shared
{
    Body q, q0, tr, cur;
    double dt_current, last_gap, last_pen, last_vn, last_toi;
    int phase, stable_count, release_count, min_dt_hits;
    double z[6], dz[6], zt[6], res[6], err, r0, Iw[9];
    double F[3], tau[3];
    double m_gap, m_pen, m_vn;
    int m_active, m_valid;
    int c_enabled, c_cleared, c_len;
    double c_tref[3];
    unsigned mask[kMaxCullLeaves / 32];
    int full;
    double Rs[9], tl[3]; // R_B^T R_A and R_B^T (r_A - r_B) of the pass's pose
    double box[6];
    double red[kMaxWarps][6];
    MinRec mins[kMaxWarps];
    int cnt[kMaxWarps][2];
    int scan[kMaxWarps];
    int flag, count, mi;
    double lo, hi, hm_pen, toi; // bisection bracket, its measure, the step
    double m0_gap;              // gap at the start of the step
    int hit, event;
    int scene;                  // index of the scene in the batch
    double alpha;               // line search
    int found;
    // rows of per-warp partial sums of the contact Jacobians (one row per
    // warp of the scene; after the reduction row 0 holds Jp then Jv)
    double* jred;
    int n_newton, n_resid, n_solves; // this launch's counts for the scene
    // (CTA per scene) per-(chunk, warp) filtered-point counts, then their
    // exclusive prefix, and the total; NULL in the warp-per-scene variant
    int* pref;
    int pref_total;
};

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ void matvec(const double R[9], const double x[3], double y[3])
{
    for (int i = 0; i < 3; ++i) y[i] = R[3 * i] * x[0] + R[3 * i + 1] * x[1] + R[3 * i + 2] * x[2];
}

__device__ __forceinline__ void matTvec(const double R[9], const double x[3], double y[3])
{
    for (int i = 0; i < 3; ++i) y[i] = R[i] * x[0] + R[3 + i] * x[1] + R[6 + i] * x[2];
}

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3])
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ double warp_dsum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ int warp_isum(int v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// The threads working on one scene: a whole CTA (Grp<false>) or one warp
// (Grp<true>, several scenes per CTA).
template <bool W>
struct Grp;

template <>
struct Grp<false>
{
    __device__ static int rank() { return (int)threadIdx.x; }
    __device__ static int size() { return (int)blockDim.x; }
    __device__ static void sync() { __syncthreads(); }
    __device__ static int count(bool f) { return __syncthreads_count(f); }
    __device__ static bool any(bool f) { return __syncthreads_or(f) != 0; }
    __device__ static int warp() { return (int)(threadIdx.x >> 5); }
    __device__ static int warps() { return (int)(blockDim.x >> 5); }
};

template <>
struct Grp<true>
{
    __device__ static int rank() { return (int)(threadIdx.x & 31); }
    __device__ static int size() { return 32; }
    __device__ static void sync() { __syncwarp(); }
    __device__ static int count(bool f) { return __popc(__ballot_sync(0xffffffffu, f)); }
    __device__ static bool any(bool f) { return __any_sync(0xffffffffu, f) != 0; }
    __device__ static int warp() { return 0; }
    __device__ static int warps() { return 1; }
};

// TrilinearSDFGrid.query_batch for one point (sdf_grid.py:138-204); with
// `hess`, also the interpolant's mixed second derivatives {xy, xz, yz} (its
// diagonal is zero).
__device__ bool sample64(const BeView& b, const double Y[3], double& g, double grad[3], double* hess = nullptr)
{
    const int n[3] = {b.g.nx, b.g.ny, b.g.nz};
    int c[3];
    double f[3];
    for (int a = 0; a < 3; ++a)
    {
        f[a] = (Y[a] - b.g.bmin[a]) / b.g.voxel[a] - 0.5;
        if (!(f[a] >= 0.0 && f[a] < (double)(n[a] - 1))) return false;
        c[a] = (int)floor(f[a]);
        if (c[a] < 0 || c[a] + 1 >= n[a]) return false;
    }
    const double uv = f[0] - c[0], vv = f[1] - c[1], wv = f[2] - c[2];
    const int64_t sy = n[0], sz = (int64_t)n[0] * n[1];
    const int64_t i0 = c[0] + sy * c[1] + sz * c[2];
    const double* phi = b.phi64;
    const double p000 = phi[i0], p100 = phi[i0 + 1], p010 = phi[i0 + sy], p110 = phi[i0 + 1 + sy];
    const double p001 = phi[i0 + sz], p101 = phi[i0 + 1 + sz], p011 = phi[i0 + sy + sz],
                 p111 = phi[i0 + 1 + sy + sz];
    const double one_u = 1.0 - uv, one_v = 1.0 - vv, one_w = 1.0 - wv;
    g = p000 * one_u * one_v * one_w + p100 * uv * one_v * one_w + p010 * one_u * vv * one_w +
        p110 * uv * vv * one_w + p001 * one_u * one_v * wv + p101 * uv * one_v * wv +
        p011 * one_u * vv * wv + p111 * uv * vv * wv;
    const double ihx = 1.0 / b.g.voxel[0], ihy = 1.0 / b.g.voxel[1], ihz = 1.0 / b.g.voxel[2];
    grad[0] = ((p100 - p000) * one_v * one_w + (p110 - p010) * vv * one_w + (p101 - p001) * one_v * wv +
               (p111 - p011) * vv * wv) * ihx;
    grad[1] = ((p010 - p000) * one_u * one_w + (p110 - p100) * uv * one_w + (p011 - p001) * one_u * wv +
               (p111 - p101) * uv * wv) * ihy;
    grad[2] = ((p001 - p000) * one_u * one_v + (p101 - p100) * uv * one_v + (p011 - p010) * one_u * vv +
               (p111 - p110) * uv * vv) * ihz;
    if (hess)
    {
        hess[0] = ((p110 - p010 - p100 + p000) * one_w + (p111 - p011 - p101 + p001) * wv) * (ihx * ihy);
        hess[1] = ((p101 - p001 - p100 + p000) * one_v + (p111 - p011 - p110 + p010) * vv) * (ihx * ihz);
        hess[2] = ((p011 - p001 - p010 + p000) * one_u + (p111 - p101 - p110 + p100) * uv) * (ihy * ihz);
    }
    return true;
}

// R_sdf = R_B^T R_A, t_sdf = R_B^T (r_A - r_B) of a pose (contacts_sdf.py:
// 275-286), thread 0.
__device__ __forceinline__ void sdf_frame(const BeView& b, const Body& s, double Rs[9], double tl[3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Rs[3 * i + j] = b.RB[i] * s.R[j] + b.RB[3 + i] * s.R[3 + j] + b.RB[6 + i] * s.R[6 + j];
    double d[3] = {s.r[0] - b.rB[0], s.r[1] - b.rB[1], s.r[2] - b.rB[2]};
    matTvec(b.RB, d, tl);
}

// Y = R_sdf X + t_sdf with the pass's frame.
__device__ __forceinline__ void to_sdf(const Shared& s, const double X[3], double Y[3])
{
    matvec(s.Rs, X, Y);
    for (int a = 0; a < 3; ++a) Y[a] = Y[a] + s.tl[a];
}

// The broad phase of evaluate / measure_pair for the pose in s.cur
// (contacts_sdf.py:244-269, bvh.py:62-80): leaf mask and the `full` flag.
template <bool W>
__device__ void broad_phase(const BeView& b, Shared& s)
{
    if (Grp<W>::rank() == 0) sdf_frame(b, s.cur, s.Rs, s.tl);
    if (!b.cull)
    {
        if (Grp<W>::rank() == 0) s.full = 1;
        Grp<W>::sync();
        return;
    }
    if (Grp<W>::rank() == 0)
    {
        double lo[3], hi[3], d[3];
        for (int a = 0; a < 3; ++a) d[a] = b.bmin[a] - s.cur.r[a];
        matTvec(s.cur.R, d, lo);
        for (int a = 0; a < 3; ++a) d[a] = b.bmax[a] - s.cur.r[a];
        matTvec(s.cur.R, d, hi);
        bool enc = true;
        for (int a = 0; a < 3; ++a)
        {
            s.box[a] = lo[a] - b.box_margin;
            s.box[3 + a] = hi[a] + b.box_margin;
            enc = enc && s.box[a] <= b.root[a] && s.box[3 + a] >= b.root[3 + a];
        }
        s.full = enc ? 1 : 0;
    }
    for (int w = Grp<W>::rank(); w < (b.nleaves + 31) / 32; w += Grp<W>::size()) s.mask[w] = 0u;
    Grp<W>::sync();
    if (s.full) return;
    bool any = false;
    for (int l = Grp<W>::rank(); l < b.nleaves; l += Grp<W>::size())
    {
        const double* x = b.leaf_box + 6 * (int64_t)l;
        const bool skip = x[3] < s.box[0] || x[4] < s.box[1] || x[5] < s.box[2] || x[0] > s.box[3] ||
                          x[1] > s.box[4] || x[2] > s.box[5];
        if (!skip)
        {
            atomicOr(&s.mask[l >> 5], 1u << (l & 31));
            any = true;
        }
    }
    const int none = Grp<W>::any(any) ? 0 : 1;
    if (Grp<W>::rank() == 0 && none) s.full = 1;
    Grp<W>::sync();
}

// Point i of the kept list in the reference's order (original order when
// every point is kept, else the stored leaf order restricted to kept
// leaves); returns whether it is kept and its coordinates / weight.
__device__ __forceinline__ bool point_at(const BeView& b, const Shared& s, int i, double X[3], double& w)
{
    if (i >= b.nq) return false;
    if (s.full)
    {
        X[0] = b.ox[3 * i];
        X[1] = b.ox[3 * i + 1];
        X[2] = b.ox[3 * i + 2];
        w = b.ow[i];
        return true;
    }
    const int l = b.pleaf[i];
    if (!((s.mask[l >> 5] >> (l & 31)) & 1u)) return false;
    X[0] = b.px[3 * i];
    X[1] = b.px[3 * i + 1];
    X[2] = b.px[3 * i + 2];
    w = b.pw[i];
    return true;
}

// Block-wide exclusive position of `flag` within the chunk; *total = count.
template <bool W>
__device__ __forceinline__ int chunk_scan(Shared& s, bool flag, int& total)
{
    const int warp = Grp<W>::warp(), lane = (int)(threadIdx.x & 31);
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) s.scan[warp] = __popc(bal);
    Grp<W>::sync();
    int off = 0;
    total = 0;
    for (int w = 0; w < Grp<W>::warps(); ++w)
    {
        off += w < warp ? s.scan[w] : 0;
        total += s.scan[w];
    }
    Grp<W>::sync();
    return off + __popc(bal & ((1u << lane) - 1u));
}

// 3x3 helpers for the Jacobian (row-major).
__device__ __forceinline__ void skew3(const double a[3], double S[9])
{
    S[0] = 0.0;
    S[1] = -a[2];
    S[2] = a[1];
    S[3] = a[2];
    S[4] = 0.0;
    S[5] = -a[0];
    S[6] = -a[1];
    S[7] = a[0];
    S[8] = 0.0;
}

__device__ __forceinline__ void mat3mul(const double A[9], const double B[9], double C[9])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// Per-point derivatives of the force law (contacts_sdf.py:329-385) for the
// exact tangent: Gt = d fq / d(material point displacement, world) at fixed
// A velocities, U = d fq / d(relative velocity u).  Inputs as in eval_pass;
// H3 = the SDF-frame mixed partials {xy, xz, yz}.
__device__ void point_jacobian(const BeView& b, const double rg[3], const double H3[3], double g, double p,
                               double gn, const double u[3], bool damp, bool fric, double phat, const double un[3],
                               const double ut[3], double den, double Gt[9], double U[9])
{
    // world Hessian Hw = RB Hs RB^T
    const double Hs[9] = {0.0, H3[0], H3[1], H3[0], 0.0, H3[2], H3[1], H3[2], 0.0};
    double T[9], Hw[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            T[3 * i + j] = b.RB[3 * i] * Hs[j] + b.RB[3 * i + 1] * Hs[3 + j] + b.RB[3 * i + 2] * Hs[6 + j];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Hw[3 * i + j] = T[3 * i] * b.RB[3 * j] + T[3 * i + 1] * b.RB[3 * j + 1] + T[3 * i + 2] * b.RB[3 * j + 2];
    const double dl = -g;
    const double pp = -b.c.stiffness * b.c.order *
                      (b.c.order == 2.0 ? dl : b.c.order == 1.0 ? 1.0 : pow(dl, b.c.order - 1.0)); // dp/dg
    const double vn = u[0] * rg[0] + u[1] * rg[1] + u[2] * rg[2];
    const double udn = u[0] * un[0] + u[1] * un[1] + u[2] * un[2];
    const double mu = b.c.friction, c = b.c.damping;
    double ag[3], B[9];
    for (int i = 0; i < 3; ++i)
    {
        ag[i] = pp * rg[i];
        if (fric) ag[i] = ag[i] - mu * gn * pp * ut[i] / den;
        for (int j = 0; j < 3; ++j)
        {
            const double I = i == j ? 1.0 : 0.0;
            B[3 * i + j] = p * I;
            if (damp) B[3 * i + j] = B[3 * i + j] - c * (rg[i] * u[j] + vn * I);
            U[3 * i + j] = damp ? -c * rg[i] * rg[j] : 0.0;
        }
    }
    if (fric)
    {
        // Mt = (I - ut ut^T / den^2) / den, P = I - un un^T
        double Mt[9], P[9], Q[9], QP[9], MQ[9], MP[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                const double I = i == j ? 1.0 : 0.0;
                Mt[3 * i + j] = (I - ut[i] * ut[j] / (den * den)) / den;
                P[3 * i + j] = I - un[i] * un[j];
                Q[3 * i + j] = udn * I + un[i] * u[j];
            }
        mat3mul(Q, P, QP);
        mat3mul(Mt, QP, MQ);
        mat3mul(Mt, P, MP);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
            {
                B[3 * i + j] = B[3 * i + j] - mu * p * ut[i] * un[j] / den + mu * p * MQ[3 * i + j];
                U[3 * i + j] = U[3 * i + j] - mu * phat * MP[3 * i + j];
            }
    }
    // G = ag rg^T + B Hw, Gt = G - U [wB]x
    double BH[9], Wb[9], UW[9];
    mat3mul(B, Hw, BH);
    skew3(b.wB, Wb);
    mat3mul(U, Wb, UW);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Gt[3 * i + j] = ag[i] * rg[j] + BH[3 * i + j] - UW[3 * i + j];
}

// Adds the point's weighted contributions to Jp and Jv into the warp's row
// (every lane of the warp calls it; inactive lanes pass w = 0).  Column by
// column: for each of the 12 columns the 6 entries are warp-summed and lane
// 0 adds them to its row in chunk order.
__device__ void add_point_jacobian(double* row, double w, const double Gt[9], const double U[9],
                                   const double off[3], const double fq[3], const double wA[3])
{
    const int lane = (int)(threadIdx.x & 31);
    double Ox[9], Wx[9], Fx[9], A[9], UW[9];
    skew3(off, Ox);
    skew3(wA, Wx);
    skew3(fq, Fx);
    // A = Gt + U [w]x, so that dfq/dtheta = -A [off]x
    mat3mul(U, Wx, UW);
    for (int k = 0; k < 9; ++k) A[k] = Gt[k] + UW[k];
#pragma unroll 1
    for (int col = 0; col < 12; ++col)
    {
        const int m = col / 6, cc = col % 6, c3 = cc % 3;
        double f[3], t[3];
        const double ox[3] = {Ox[c3], Ox[3 + c3], Ox[6 + c3]}; // column c3 of [off]x
        if (m == 0 && cc < 3)
            for (int i = 0; i < 3; ++i) f[i] = Gt[3 * i + c3];
        else if (m == 0)
            for (int i = 0; i < 3; ++i) f[i] = -(A[3 * i] * ox[0] + A[3 * i + 1] * ox[1] + A[3 * i + 2] * ox[2]);
        else if (cc < 3)
            for (int i = 0; i < 3; ++i) f[i] = U[3 * i + c3];
        else
            for (int i = 0; i < 3; ++i) f[i] = -(U[3 * i] * ox[0] + U[3 * i + 1] * ox[1] + U[3 * i + 2] * ox[2]);
        for (int i = 0; i < 3; ++i) t[i] = Ox[3 * i] * f[0] + Ox[3 * i + 1] * f[1] + Ox[3 * i + 2] * f[2];
        if (m == 0 && cc >= 3)
            for (int i = 0; i < 3; ++i)
                t[i] = t[i] + (Fx[3 * i] * ox[0] + Fx[3 * i + 1] * ox[1] + Fx[3 * i + 2] * ox[2]);
        for (int i = 0; i < 3; ++i)
        {
            const double vf = warp_dsum(w * f[i]);
            const double vt = warp_dsum(w * t[i]);
            if (lane == 0)
            {
                row[36 * m + 6 * i + cc] += vf;
                row[36 * m + 6 * (3 + i) + cc] += vt;
            }
        }
    }
}

// SDFContactEngine.evaluate for s.cur with the cache (F, tau into shared);
// JAC: also Jp and Jv (row 0 of s.jred) for the exact tangent.
template <bool W, bool JAC>
__device__ void eval_pass(const BeView& b, Shared& s)
{
    broad_phase<W>(b, s);
    const double narrow = b.cull ? b.narrow : INFINITY;
    const int warp = Grp<W>::warp(), lane = (int)(threadIdx.x & 31);
    double* jrow = JAC ? s.jred + kJac * warp : nullptr;
    if (JAC && lane == 0)
        for (int e = 0; e < kJac; ++e) jrow[e] = 0.0;
    // the number of narrow-filtered points decides whether the cache is used
    const int nw = Grp<W>::warps();
    const bool fast = !W && ((b.nq + Grp<W>::size() - 1) / Grp<W>::size()) * nw <= kPrefCap;
    const unsigned lt = (1u << lane) - 1u;
    int L = 0;
    if (fast)
    {
        // counts per (chunk, warp), no barrier in the loop
        for (int c0 = 0, k = 0; c0 < b.nq; c0 += Grp<W>::size(), ++k)
        {
            double X[3], w, Y[3];
            bool f = false;
            if (point_at(b, s, c0 + Grp<W>::rank(), X, w))
            {
                to_sdf(s, X, Y);
                f = fabs(Y[2]) < narrow;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, f);
            if (lane == 0) s.pref[k * nw + warp] = __popc(bal);
        }
        Grp<W>::sync();
        if (warp == 0)
        {
            // exclusive prefix in (chunk, warp) order = point order
            const int E = ((b.nq + Grp<W>::size() - 1) / Grp<W>::size()) * nw;
            int carry = 0;
            for (int e0 = 0; e0 < E; e0 += 32)
            {
                const int e = e0 + lane;
                const int v = e < E ? s.pref[e] : 0;
                int x = v;
                for (int o = 1; o < 32; o <<= 1)
                {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                if (e < E) s.pref[e] = carry + x - v;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
            if (lane == 0) s.pref_total = carry;
        }
        Grp<W>::sync();
        L = s.pref_total;
    }
    else
    {
        for (int c0 = 0; c0 < b.nq; c0 += Grp<W>::size())
        {
            double X[3], w, Y[3];
            bool f = false;
            if (point_at(b, s, c0 + Grp<W>::rank(), X, w))
            {
                to_sdf(s, X, Y);
                f = fabs(Y[2]) < narrow;
            }
            L += Grp<W>::count(f);
        }
    }
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (L > 0)
    {
        const bool use = s.c_enabled && !s.c_cleared && s.c_len >= 0 && L == s.c_len;
        const bool store = !use && s.c_enabled;
        double tsdf[3], d[3] = {s.cur.r[0] - b.rB[0], s.cur.r[1] - b.rB[1], s.cur.r[2] - b.rB[2]};
        matTvec(b.RB, d, tsdf);
        const int64_t base_c = (int64_t)s.scene * b.nq;
        int base = 0;
        for (int c0 = 0, k = 0; c0 < b.nq; c0 += Grp<W>::size(), ++k)
        {
            double X[3], w = 0.0, Y[3];
            bool f = false;
            if (point_at(b, s, c0 + Grp<W>::rank(), X, w))
            {
                to_sdf(s, X, Y);
                f = fabs(Y[2]) < narrow;
            }
            int pos;
            if (fast)
            {
                // the same flags as the counting loop: position from the prefix
                pos = s.pref[k * nw + warp] + __popc(__ballot_sync(0xffffffffu, f) & lt);
            }
            else
            {
                int total;
                pos = base + chunk_scan<W>(s, f, total);
                base += total;
            }
            bool act = false;
            double fq[3] = {0.0, 0.0, 0.0}, off[3] = {0.0, 0.0, 0.0};
            double Gt[9], U[9];
            if (f)
            {
                double g, gr[3], H3[3] = {0.0, 0.0, 0.0};
                bool valid;
                const int64_t ci = base_c + pos;
                if (use)
                {
                    const double dt3[3] = {tsdf[0] - s.c_tref[0], tsdf[1] - s.c_tref[1], tsdf[2] - s.c_tref[2]};
                    gr[0] = b.cgrad[3 * ci];
                    gr[1] = b.cgrad[3 * ci + 1];
                    gr[2] = b.cgrad[3 * ci + 2];
                    g = b.cg[ci] + (gr[0] * dt3[0] + gr[1] * dt3[1] + gr[2] * dt3[2]);
                    valid = b.cvalid[ci] != 0;
                }
                else
                {
                    valid = sample64(b, Y, g, gr, JAC ? H3 : nullptr);
                    if (!valid)
                    {
                        g = 0.0;
                        gr[0] = gr[1] = gr[2] = 0.0;
                    }
                    if (store)
                    {
                        b.cg[ci] = g;
                        b.cgrad[3 * ci] = gr[0];
                        b.cgrad[3 * ci + 1] = gr[1];
                        b.cgrad[3 * ci + 2] = gr[2];
                        b.cvalid[ci] = valid ? 1 : 0;
                    }
                }
                const double delta = -g > 0.0 ? -g : 0.0;
                const double p = b.c.stiffness *
                                 (b.c.order == 2.0 ? delta * delta : b.c.order == 1.0 ? delta : pow(delta, b.c.order));
                if (valid && p > 1e-30)
                {
                    act = true;
                    // force law (contacts_sdf.py:329-385)
                    double rg[3], xw[3], uA[3], uB[3], u[3], t3[3];
                    matvec(b.RB, gr, rg);
                    const double gn = sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
                    matvec(s.cur.R, X, off);
                    for (int a = 0; a < 3; ++a) xw[a] = s.cur.r[a] + off[a];
                    for (int a = 0; a < 3; ++a) fq[a] = p * rg[a];
                    const double phat = p * gn;
                    cross3(s.cur.w, off, t3);
                    for (int a = 0; a < 3; ++a) uA[a] = s.cur.v[a] + t3[a];
                    double offB[3] = {xw[0] - b.rB[0], xw[1] - b.rB[1], xw[2] - b.rB[2]};
                    cross3(b.wB, offB, t3);
                    for (int a = 0; a < 3; ++a) uB[a] = b.vB[a] + t3[a];
                    for (int a = 0; a < 3; ++a) u[a] = uA[a] - uB[a];
                    const bool damp = b.c.damping > 0.0 && g < 0.0;
                    if (damp)
                    {
                        const double vn = u[0] * rg[0] + u[1] * rg[1] + u[2] * rg[2];
                        for (int a = 0; a < 3; ++a) fq[a] = fq[a] + b.c.damping * (-vn) * rg[a];
                    }
                    const double gs = gn > 1e-30 ? gn : 1e-30;
                    double un[3] = {rg[0] / gs, rg[1] / gs, rg[2] / gs};
                    const double udn = u[0] * un[0] + u[1] * un[1] + u[2] * un[2];
                    double ut[3] = {u[0] - udn * un[0], u[1] - udn * un[1], u[2] - udn * un[2]};
                    const double utn = sqrt(ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2]);
                    const double den = sqrt(utn * utn + b.c.regularizer * b.c.regularizer);
                    const bool fric = b.c.friction * phat > 0.0;
                    if (fric)
                        for (int a = 0; a < 3; ++a) fq[a] = fq[a] + -b.c.friction * phat * ut[a] / den;
                    double tq[3];
                    cross3(off, fq, tq);
                    for (int a = 0; a < 3; ++a)
                    {
                        acc[a] += w * fq[a];
                        acc[3 + a] += w * tq[a];
                    }
                    if (JAC) point_jacobian(b, rg, H3, g, p, gn, u, damp, fric, phat, un, ut, den, Gt, U);
                }
            }
            if (JAC && __any_sync(0xffffffffu, act))
            {
                if (!act)
                    for (int k = 0; k < 9; ++k) Gt[k] = U[k] = 0.0;
                add_point_jacobian(jrow, act ? w : 0.0, Gt, U, off, fq, s.cur.w);
            }
        }
        if (Grp<W>::rank() == 0 && store)
        {
            for (int a = 0; a < 3; ++a) s.c_tref[a] = tsdf[a];
            s.c_len = L;
            s.c_cleared = 0;
        }
    }
    for (int q = 0; q < 6; ++q)
    {
        const double v = warp_dsum(acc[q]);
        if (lane == 0) s.red[warp][q] = v;
    }
    Grp<W>::sync();
    if (Grp<W>::rank() == 0)
    {
        for (int q = 0; q < 6; ++q)
        {
            double v = 0.0;
            for (int w = 0; w < Grp<W>::warps(); ++w) v += s.red[w][q];
            if (q < 3)
                s.F[q] = v;
            else
                s.tau[q - 3] = v;
        }
        if (JAC)
            for (int wp = 1; wp < Grp<W>::warps(); ++wp)
                for (int e = 0; e < kJac; ++e) s.jred[e] += s.jred[kJac * wp + e];
    }
    Grp<W>::sync();
}

// measure_pair for s.cur (contacts_sdf.py:171-214): m_gap, m_pen, m_vn,
// m_active, m_valid.
template <bool W>
__device__ void measure_pass(const BeView& b, Shared& s)
{
    broad_phase<W>(b, s);
    MinRec best{INFINITY, INT_MAX, -1};
    int nv = 0, na = 0;
    // ties of the minimum go to the first kept point; the list index orders
    // kept points as their positions among the kept points do, so it serves
    // as the key and the loop needs no block scan
    for (int c0 = 0; c0 < b.nq; c0 += Grp<W>::size())
    {
        double X[3], w, Y[3];
        const int i = c0 + Grp<W>::rank();
        if (!point_at(b, s, i, X, w)) continue;
        to_sdf(s, X, Y);
        double g, gr[3];
        if (!sample64(b, Y, g, gr)) continue;
        ++nv;
        if (g < 0.0) ++na;
        if (g < best.gap || (g == best.gap && i < best.key)) best = MinRec{g, i, i};
    }
    const int warp = Grp<W>::warp(), lane = (int)(threadIdx.x & 31);
    for (int o = 16; o > 0; o >>= 1)
    {
        MinRec q;
        q.gap = __shfl_down_sync(0xffffffffu, best.gap, o);
        q.key = __shfl_down_sync(0xffffffffu, best.key, o);
        q.i = __shfl_down_sync(0xffffffffu, best.i, o);
        if (q.gap < best.gap || (q.gap == best.gap && q.key < best.key)) best = q;
    }
    nv = warp_isum(nv);
    na = warp_isum(na);
    if (lane == 0)
    {
        s.mins[warp] = best;
        s.cnt[warp][0] = nv;
        s.cnt[warp][1] = na;
    }
    Grp<W>::sync();
    if (Grp<W>::rank() == 0)
    {
        MinRec m = s.mins[0];
        int v = s.cnt[0][0], a = s.cnt[0][1];
        for (int k = 1; k < Grp<W>::warps(); ++k)
        {
            if (s.mins[k].gap < m.gap || (s.mins[k].gap == m.gap && s.mins[k].key < m.key)) m = s.mins[k];
            v += s.cnt[k][0];
            a += s.cnt[k][1];
        }
        s.m_valid = v;
        s.m_active = a;
        s.m_gap = v ? m.gap : INFINITY;
        s.m_pen = v && m.gap < 0.0 ? -m.gap : 0.0;
        s.m_vn = 0.0;
        s.count = v ? m.key : -1; // the minimum's point index
        s.mi = v ? m.i : -1;
    }
    Grp<W>::sync();
    // normal relative velocity at the minimum point (contacts_sdf.py:199-211)
    if (Grp<W>::rank() == 0 && s.mi >= 0)
    {
        double X[3], w, Y[3], g, gr[3];
        point_at(b, s, s.mi, X, w);
        to_sdf(s, X, Y);
        sample64(b, Y, g, gr);
        const double gn = sqrt(gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
        double un[3] = {0.0, 0.0, 1.0};
        if (gn > 1e-30)
            for (int a = 0; a < 3; ++a) un[a] = gr[a] / gn;
        double n[3];
        matvec(b.RB, un, n);
        const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (nn > 1e-30)
            for (int a = 0; a < 3; ++a) n[a] = n[a] / nn;
        double off[3], xw[3], t3[3], uA[3], uB[3];
        matvec(s.cur.R, X, off);
        for (int a = 0; a < 3; ++a) xw[a] = s.cur.r[a] + off[a];
        cross3(s.cur.w, off, t3);
        for (int a = 0; a < 3; ++a) uA[a] = s.cur.v[a] + t3[a];
        double offB[3] = {xw[0] - b.rB[0], xw[1] - b.rB[1], xw[2] - b.rB[2]};
        cross3(b.wB, offB, t3);
        for (int a = 0; a < 3; ++a) uB[a] = b.vB[a] + t3[a];
        double du[3] = {uA[0] - uB[0], uA[1] - uB[1], uA[2] - uB[2]};
        s.m_vn = dot3(du, n);
    }
    Grp<W>::sync();
}

// _kinematic_update (implicit_be.py:507-534), thread 0.
__device__ void kinematic(const Body& q0, const double V[6], double dt, Body& out)
{
    for (int a = 0; a < 3; ++a)
    {
        out.v[a] = V[a];
        out.w[a] = V[3 + a];
        out.r[a] = q0.r[a] + dt * V[a];
    }
    const double th[3] = {dt * V[3], dt * V[4], dt * V[5]};
    const double n = sqrt(th[0] * th[0] + th[1] * th[1] + th[2] * th[2]);
    if (n > 1e-30)
    {
        const double ax[3] = {th[0] / n, th[1] / n, th[2] / n};
        const double c = cos(n), sn = sin(n);
        const double K[9] = {0.0, -ax[2], ax[1], ax[2], 0.0, -ax[0], -ax[1], ax[0], 0.0};
        double dR[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                dR[3 * i + j] = (i == j ? c : 0.0) + sn * K[3 * i + j] + (1.0 - c) * (ax[i] * ax[j]);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                out.R[3 * i + j] = dR[3 * i] * q0.R[j] + dR[3 * i + 1] * q0.R[3 + j] + dR[3 * i + 2] * q0.R[6 + j];
    }
    else
    {
        for (int k = 0; k < 9; ++k) out.R[k] = q0.R[k];
    }
    out.t = q0.t;
}

// _residual at V = z (implicit_be.py:536-604): s.res, s.err, s.Iw, s.cur;
// JAC: also the contact Jacobians of the exact tangent (s.jred).
template <bool W, bool JAC>
__device__ void residual(const BeView& b, Shared& s, const double* z, double dt, bool allowed)
{
    if (Grp<W>::rank() == 0)
    {
        kinematic(s.q0, z, dt, s.cur);
        s.n_resid += 1;
    }
    Grp<W>::sync();
    if (allowed) eval_pass<W, JAC>(b, s);
    if (Grp<W>::rank() == 0)
    {
        double RI[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                RI[3 * i + j] = s.cur.R[3 * i] * b.Ib[j] + s.cur.R[3 * i + 1] * b.Ib[3 + j] + s.cur.R[3 * i + 2] * b.Ib[6 + j];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                s.Iw[3 * i + j] = RI[3 * i] * s.cur.R[3 * j] + RI[3 * i + 1] * s.cur.R[3 * j + 1] +
                                  RI[3 * i + 2] * s.cur.R[3 * j + 2];
        double dV[6];
        dV[0] = z[0] - s.q0.v[0];
        dV[1] = z[1] - s.q0.v[1];
        dV[2] = z[2] - s.q0.v[2];
        dV[3] = z[3] - s.q0.w[0];
        dV[4] = z[4] - s.q0.w[1];
        dV[5] = z[5] - s.q0.w[2];
        double Iww[3], C[3];
        matvec(s.Iw, s.cur.w, Iww);
        cross3(s.cur.w, Iww, C);
        double err = 0.0;
        for (int a = 0; a < 3; ++a)
        {
            double Q = b.mass * b.gravity[a];
            if (allowed) Q = Q + s.F[a];
            s.res[a] = b.mass * dV[a] / dt + 0.0 - Q;
        }
        for (int a = 0; a < 3; ++a)
        {
            const double MdV = s.Iw[3 * a] * dV[3] + s.Iw[3 * a + 1] * dV[4] + s.Iw[3 * a + 2] * dV[5];
            double Q = 0.0;
            if (allowed) Q = Q + s.tau[a];
            s.res[3 + a] = MdV / dt + C[a] - Q;
        }
        for (int a = 0; a < 6; ++a) err = fmax(err, fabs(s.res[a]));
        s.err = err;
    }
    Grp<W>::sync();
}

// Left Jacobian of SO(3): exp(phi + d) = exp([J_l(phi) d]x) exp(phi) + O(d^2).
__device__ void left_jacobian(const double phi[3], double J[9])
{
    const double t = sqrt(phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2]);
    double a, c;
    if (t < 1e-4)
    {
        a = 0.5 - t * t / 24.0;
        c = 1.0 / 6.0 - t * t / 120.0;
    }
    else
    {
        a = (1.0 - cos(t)) / (t * t);
        c = (t - sin(t)) / (t * t * t);
    }
    double S[9], S2[9];
    skew3(phi, S);
    mat3mul(S, S, S2);
    for (int k = 0; k < 9; ++k) J[k] = (k % 4 == 0 ? 1.0 : 0.0) + a * S[k] + c * S2[k];
}

// The exact tangent dR/dV at the state of the last residual (s.cur, s.Iw,
// s.jred) and the Newton step s.dz = -K^-1 res; thread 0.  Returns false
// when K is singular (no usable pivot).
__device__ bool exact_newton_step(const BeView& b, Shared& s, double dt, bool allowed)
{
    double K[36];
    for (int k = 0; k < 36; ++k) K[k] = 0.0;
    for (int a = 0; a < 3; ++a) K[7 * a] = b.mass / dt;
    const double* w = s.cur.w;
    double dw[3] = {w[0] - s.q0.w[0], w[1] - s.q0.w[1], w[2] - s.q0.w[2]};
    const double phi[3] = {dt * w[0], dt * w[1], dt * w[2]};
    double Jl[9], Iw_dw[3], Iw_w[3], S1[9], S2[9], S3[9], S4[9], A1[9], A2[9], A3[9], T1[9], T3[9];
    left_jacobian(phi, Jl);
    matvec(s.Iw, dw, Iw_dw);
    matvec(s.Iw, w, Iw_w);
    // A1 = -[Iw dw]x + Iw [dw]x (inertia term through R(w))
    skew3(Iw_dw, S1);
    skew3(dw, S2);
    mat3mul(s.Iw, S2, T1);
    for (int k = 0; k < 9; ++k) A1[k] = -S1[k] + T1[k];
    // A2 = -[Iw w]x + [w]x Iw (gyroscopic term, explicit w)
    skew3(Iw_w, S3);
    skew3(w, S4);
    mat3mul(S4, s.Iw, T1);
    for (int k = 0; k < 9; ++k) A2[k] = -S3[k] + T1[k];
    // A3 = h [w]x (-[Iw w]x + Iw [w]x) (gyroscopic term through R(w))
    mat3mul(s.Iw, S4, T1);
    for (int k = 0; k < 9; ++k) T1[k] = -S3[k] + T1[k];
    mat3mul(S4, T1, T3);
    for (int k = 0; k < 9; ++k) A3[k] = dt * T3[k];
    double B[9];
    for (int k = 0; k < 9; ++k) B[k] = A1[k] + A3[k];
    mat3mul(B, Jl, T1);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) K[6 * (3 + i) + 3 + j] = s.Iw[3 * i + j] / dt + T1[3 * i + j] + A2[3 * i + j];
    if (allowed)
    {
        // K -= Jv + Jp diag(h I, h J_l)
        const double* Jp = s.jred;
        const double* Jv = s.jred + 36;
        for (int i = 0; i < 6; ++i)
        {
            for (int j = 0; j < 3; ++j) K[6 * i + j] = K[6 * i + j] - (Jv[6 * i + j] + dt * Jp[6 * i + j]);
            for (int j = 0; j < 3; ++j)
            {
                const double jr = Jp[6 * i + 3] * Jl[j] + Jp[6 * i + 4] * Jl[3 + j] + Jp[6 * i + 5] * Jl[6 + j];
                K[6 * i + 3 + j] = K[6 * i + 3 + j] - (Jv[6 * i + 3 + j] + dt * jr);
            }
        }
    }
    // Gaussian elimination with partial pivoting on [K | -res]
    double x[6];
    for (int a = 0; a < 6; ++a) x[a] = -s.res[a];
    for (int c = 0; c < 6; ++c)
    {
        int piv = c;
        for (int r = c + 1; r < 6; ++r)
            if (fabs(K[6 * r + c]) > fabs(K[6 * piv + c])) piv = r;
        if (!(fabs(K[6 * piv + c]) > 0.0)) return false;
        if (piv != c)
        {
            for (int j = 0; j < 6; ++j)
            {
                const double t = K[6 * c + j];
                K[6 * c + j] = K[6 * piv + j];
                K[6 * piv + j] = t;
            }
            const double t = x[c];
            x[c] = x[piv];
            x[piv] = t;
        }
        for (int r = c + 1; r < 6; ++r)
        {
            const double f = K[6 * r + c] / K[6 * c + c];
            for (int j = c; j < 6; ++j) K[6 * r + j] = K[6 * r + j] - f * K[6 * c + j];
            x[r] = x[r] - f * x[c];
        }
    }
    for (int c = 5; c >= 0; --c)
    {
        double v = x[c];
        for (int j = c + 1; j < 6; ++j) v = v - K[6 * c + j] * x[j];
        x[c] = v / K[6 * c + c];
    }
    for (int a = 0; a < 6; ++a) s.dz[a] = x[a];
    return true;
}

// _step_be (implicit_be.py:468-505): src -> dst (thread-0 copies), contact
// forces of the pair when `allowed`.  EXACT: exact contact every residual
// and the analytic tangent (see the file comment).
template <bool W, bool EXACT>
__device__ void step_be(const BeView& b, Shared& s, const Body* src, Body* dst, double dt, bool allowed)
{
    if (Grp<W>::rank() == 0)
    {
        s.q0 = *src;
        for (int a = 0; a < 3; ++a)
        {
            s.z[a] = src->v[a];
            s.z[3 + a] = src->w[a];
        }
        s.c_enabled = (allowed && !EXACT) ? 1 : 0;
        s.c_cleared = 1;
        s.n_solves += 1;
    }
    Grp<W>::sync();
    residual<W, EXACT>(b, s, s.z, dt, allowed);
    for (int it = 0; it < b.p.max_iter; ++it)
    {
        if (s.err < b.p.tol) break;
        if (Grp<W>::rank() == 0 && EXACT)
        {
            s.n_newton += 1;
            if (!exact_newton_step(b, s, dt, allowed))
                for (int a = 0; a < 6; ++a) s.dz[a] = 0.0;
            double nr = 0.0;
            for (int a = 0; a < 6; ++a) nr += s.res[a] * s.res[a];
            s.r0 = sqrt(nr);
            s.found = 0;
            s.alpha = 1.0;
        }
        else if (Grp<W>::rank() == 0)
        {
            s.n_newton += 1;
            // tangent (_tangent / _contact_tangent): M/h + diag(Kc) on the
            // translational rows; the two diagonal blocks solved exactly
            double ktt = b.mass / dt;
            double kd[3] = {ktt, ktt, ktt};
            if (allowed)
            {
                const double vel = sqrt(s.cur.v[0] * s.cur.v[0] + s.cur.v[1] * s.cur.v[1] + s.cur.v[2] * s.cur.v[2]);
                const double de = fmax(vel * dt, 1e-10);
                double stiff;
                if (b.c.order == 1.0)
                    stiff = b.c.stiffness * dt;
                else
                    stiff = b.c.stiffness * b.c.order * pow(de, b.c.order - 1.0) * dt + 5e2;
                const double tot = stiff + b.c.damping * b.area;
                for (int a = 0; a < 3; ++a) kd[a] = kd[a] + tot;
            }
            for (int a = 0; a < 3; ++a) s.dz[a] = -s.res[a] / kd[a];
            // (Iw/h) x = -res_w by Cholesky
            double A[9];
            for (int k = 0; k < 9; ++k) A[k] = s.Iw[k] / dt;
            const double l00 = sqrt(A[0]);
            const double l10 = A[3] / l00, l20 = A[6] / l00;
            const double l11 = sqrt(A[4] - l10 * l10);
            const double l21 = (A[7] - l20 * l10) / l11;
            const double l22 = sqrt(A[8] - l20 * l20 - l21 * l21);
            const double r0 = -s.res[3], r1 = -s.res[4], r2 = -s.res[5];
            const double y0 = r0 / l00, y1 = (r1 - l10 * y0) / l11, y2 = (r2 - l20 * y0 - l21 * y1) / l22;
            const double x2 = y2 / l22, x1 = (y1 - l21 * x2) / l11, x0 = (y0 - l10 * x1 - l20 * x2) / l00;
            s.dz[3] = x0;
            s.dz[4] = x1;
            s.dz[5] = x2;
            double nr = 0.0;
            for (int a = 0; a < 6; ++a) nr += s.res[a] * s.res[a];
            s.r0 = sqrt(nr);
            s.found = 0;
            s.alpha = 1.0;
        }
        Grp<W>::sync();
        if (b.p.line_search)
        {
            const double alphas[5] = {1.0, 0.5, 0.25, 0.125, 0.0625};
            for (int k = 0; k < 5; ++k)
            {
                if (Grp<W>::rank() < 6) s.zt[Grp<W>::rank()] = s.z[Grp<W>::rank()] + alphas[k] * s.dz[Grp<W>::rank()];
                Grp<W>::sync();
                residual<W, false>(b, s, s.zt, dt, allowed);
                if (Grp<W>::rank() == 0)
                {
                    double nr = 0.0;
                    for (int a = 0; a < 6; ++a) nr += s.res[a] * s.res[a];
                    if (sqrt(nr) < s.r0)
                    {
                        s.alpha = alphas[k];
                        s.found = 1;
                    }
                }
                Grp<W>::sync();
                if (s.found) break;
            }
        }
        if (Grp<W>::rank() == 0)
        {
            const double alpha = s.found ? s.alpha : 1.0;
            for (int a = 0; a < 6; ++a) s.z[a] = s.z[a] + alpha * s.dz[a];
        }
        Grp<W>::sync();
        residual<W, EXACT>(b, s, s.z, dt, allowed);
    }
    if (Grp<W>::rank() == 0)
    {
        Body out;
        kinematic(s.q0, s.z, dt, out);
        out.t = s.q0.t + dt;
        *dst = out;
        s.c_enabled = 0;
        s.c_cleared = 1;
    }
    Grp<W>::sync();
}

template <bool W>
__device__ void measure_body(const BeView& b, Shared& s, const Body& body)
{
    if (Grp<W>::rank() == 0) s.cur = body;
    Grp<W>::sync();
    measure_pass<W>(b, s);
}

__device__ __forceinline__ bool region_active(int ph)
{
    return ph == kImpacting || ph == kActive || ph == kStable || ph == kLeaving;
}

// _refresh_contact_states (implicit_be.py:248-295), thread 0, after a
// measure of the new state.
__device__ void refresh(const BeView& b, Shared& s)
{
    const sdfo_be_params& p = b.p;
    const double old = s.last_pen;
    s.last_gap = s.m_gap;
    s.last_pen = s.m_pen;
    s.last_vn = s.m_vn;
    if (s.phase == kInactive) return;
    const double release_gap = fmax(5.0 * p.pen_max, 1e-9);
    if (s.m_gap > release_gap && s.m_vn >= -1e-5)
    {
        s.release_count += 1;
        s.phase = kLeaving;
        s.dt_current = fmin(p.dt_normal, fmax(s.dt_current * p.dt_growth, p.dt_contact));
        if (s.release_count >= p.release_steps)
        {
            s.phase = kInactive;
            s.dt_current = p.dt_normal;
            s.stable_count = s.release_count = s.min_dt_hits = 0;
            s.last_toi = INFINITY;
        }
        return;
    }
    s.release_count = 0;
    if (s.phase == kImpacting)
    {
        s.phase = kActive;
        s.dt_current = fmax(p.dt_contact, p.dt_min);
        return;
    }
    const double change = fabs(s.m_pen - old);
    const double base = fmax(fabs(old), p.pen_max);
    const bool stable_pen = change <= p.pen_max || change / base <= 5e-2;
    const bool stable_vn = fabs(s.m_vn) <= 1e-5;
    if (s.m_active > 0 && stable_pen && stable_vn)
        s.stable_count += 1;
    else
        s.stable_count = 0;
    if (s.stable_count >= p.stable_steps)
    {
        s.phase = kStable;
        s.dt_current = fmin(fmin(p.dt_max_contact, p.dt_normal), fmax(s.dt_current * p.dt_growth, p.dt_contact));
    }
    else
    {
        s.phase = kActive;
        s.dt_current = fmax(p.dt_contact, p.dt_min);
    }
}

// Dynamic shared memory of the exact-tangent kernels: T / 32 rows of kJac.
template <int T>
constexpr int jac_smem_bytes() { return (T / 32) * kJac * (int)sizeof(double); }

// T threads per CTA; W: one warp per scene (T / 32 scenes per CTA), else
// the whole CTA on one scene.
template <int T, bool W, bool EXACT>
__global__ void __launch_bounds__(T, (W || T == 256) ? 3 : 4) k_be_step(BeView b, sdfo_be_scene* __restrict__ scenes, int n,
                                                const double* __restrict__ dt_req, double* __restrict__ h_out,
                                                const double* __restrict__ t_end, double dt_max,
                                                int* __restrict__ unfinished)
{
    __shared__ Shared shared_scenes[W ? T / 32 : 1];
    __shared__ int pref_table[W ? 1 : kPrefCap];
    // exact tangent: one row of Jacobian partial sums per warp, in dynamic
    // shared memory (jac_smem_bytes<T>(); the warp-per-scene variant's static
    // state alone nearly fills the 48 KB static limit)
    extern __shared__ double jred_rows[];
    const int sc = W ? (int)(blockIdx.x * (T / 32) + (threadIdx.x >> 5)) : (int)blockIdx.x;
    if (sc >= n) return; // (warps) whole warps past the last scene
    Shared& s = shared_scenes[W ? (threadIdx.x >> 5) : 0];
    const sdfo_be_params& p = b.p;
    if (Grp<W>::rank() == 0)
    {
        s.jred = EXACT ? jred_rows + (W ? (int)(threadIdx.x >> 5) * kJac : 0) : nullptr;
        s.pref = W ? nullptr : pref_table;
        s.n_newton = s.n_resid = s.n_solves = 0;
        s.scene = sc;
        const sdfo_be_scene& in = scenes[sc];
        for (int a = 0; a < 3; ++a)
        {
            s.q.r[a] = in.body.r[a];
            s.q.v[a] = in.body.v[a];
            s.q.w[a] = in.body.w[a];
        }
        for (int k = 0; k < 9; ++k) s.q.R[k] = in.body.R[k];
        s.q.t = in.t;
        s.dt_current = in.dt_current;
        s.last_gap = in.last_gap;
        s.last_pen = in.last_penetration;
        s.last_vn = in.last_normal_velocity;
        s.last_toi = in.last_toi;
        s.phase = in.phase;
        s.stable_count = in.stable_count;
        s.release_count = in.release_count;
        s.min_dt_hits = in.min_dt_hits;
        s.c_enabled = 0;
        s.c_cleared = 1;
        s.c_len = -1;
        s.event = 0;
    }
    Grp<W>::sync();
    // integrate mode (implicit_be.py:121-122): while t < t_end - 1e-15, a
    // step of at most min(dt, t_end - t); otherwise the requested step
    const double dt = t_end ? (s.q.t < t_end[sc] - 1e-15 ? fmin(dt_max, t_end[sc] - s.q.t) : 0.0) : dt_req[sc];
    if (!(dt > 0.0))
    {
        if (Grp<W>::rank() == 0 && h_out) h_out[sc] = 0.0;
        return; // nothing to do for this scene (finished)
    }
    // _activate_initially_penetrating_regions
    measure_body<W>(b, s, s.q);
    if (Grp<W>::rank() == 0)
    {
        s.last_gap = s.m_gap;
        s.last_pen = s.m_pen;
        s.last_vn = s.m_vn;
        s.m0_gap = s.m_gap;
        if (s.phase == kInactive && s.m_gap <= 0.0)
        {
            s.phase = kImpacting;
            s.dt_current = fmin(p.dt_impact, p.dt_contact);
        }
        s.toi = fmin(dt, region_active(s.phase) ? s.dt_current : p.dt_normal); // h_cap
    }
    Grp<W>::sync();
    const double h_cap = s.toi;
    // _find_earliest_new_contact
    if (s.phase == kInactive && h_cap > 0.0)
    {
        step_be<W, EXACT>(b, s, &s.q, &s.tr, h_cap, false);
        measure_body<W>(b, s, s.tr);
        if (Grp<W>::rank() == 0)
            s.flag = (s.m0_gap > 0.0 && (s.m_gap <= 0.0 || s.m_pen > p.pen_max)) ? 1 : 0;
        Grp<W>::sync();
        if (s.flag)
        {
            // _bisect_toi_pair
            if (Grp<W>::rank() == 0)
            {
                s.lo = 0.0;
                s.hi = h_cap;
                s.hm_pen = s.m_pen;
                s.hit = 0;
            }
            Grp<W>::sync();
            for (int it = 0; it < p.max_toi_bisect_iter; ++it)
            {
                if (Grp<W>::rank() == 0 && s.hi - s.lo <= p.dt_min) s.hit = 1;
                Grp<W>::sync();
                if (s.hit) break;
                const double mid = 0.5 * (s.lo + s.hi);
                step_be<W, EXACT>(b, s, &s.q, &s.tr, mid, false);
                measure_body<W>(b, s, s.tr);
                if (Grp<W>::rank() == 0)
                {
                    if (s.m_gap <= 0.0 || s.m_pen > p.pen_max)
                    {
                        s.hi = mid;
                        s.hm_pen = s.m_pen;
                    }
                    else
                        s.lo = mid;
                }
                Grp<W>::sync();
            }
            if (s.hi < p.dt_min && h_cap >= p.dt_min)
            {
                if (Grp<W>::rank() == 0)
                {
                    s.hi = p.dt_min;
                    s.hit = 1;
                }
                Grp<W>::sync();
                step_be<W, EXACT>(b, s, &s.q, &s.tr, s.hi, false);
                measure_body<W>(b, s, s.tr);
                if (Grp<W>::rank() == 0) s.hm_pen = s.m_pen;
                Grp<W>::sync();
            }
            if (Grp<W>::rank() == 0 && s.hi > 0.0)
            {
                if (s.hm_pen > p.pen_max && !s.hit)
                {
                    s.hi = fmax(s.lo, fmin(s.hi, p.dt_min));
                    s.hit = 1;
                }
                s.toi = fmin(s.hi, h_cap);
                s.event = 1;
            }
            Grp<W>::sync();
        }
    }
    double h;
    if (s.event)
    {
        h = s.toi;
        step_be<W, EXACT>(b, s, &s.q, &s.q, h, region_active(s.phase));
        if (Grp<W>::rank() == 0)
        {
            s.phase = kImpacting;
            s.dt_current = fmin(p.dt_impact, p.dt_contact);
            s.last_toi = h;
            if (s.hit) s.min_dt_hits += 1;
        }
        Grp<W>::sync();
        measure_body<W>(b, s, s.q);
        if (Grp<W>::rank() == 0)
        {
            s.last_gap = s.m_gap;
            s.last_pen = s.m_pen;
            s.last_vn = s.m_vn;
        }
    }
    else
    {
        h = h_cap;
        step_be<W, EXACT>(b, s, &s.q, &s.q, h, region_active(s.phase));
        measure_body<W>(b, s, s.q);
        if (Grp<W>::rank() == 0) refresh(b, s);
    }
    Grp<W>::sync();
    if (t_end && !(h > 0.0))
    {
        // the integrate loop's zero-progress fail-safe (implicit_be.py:124-127):
        // one plain BE step of min(dt_min, t_end - t), nothing re-measured
        h = fmin(p.dt_min, t_end[sc] - s.q.t);
        step_be<W, EXACT>(b, s, &s.q, &s.q, h, region_active(s.phase));
        Grp<W>::sync();
    }
    if (Grp<W>::rank() == 0)
    {
        sdfo_be_scene& out = scenes[sc];
        for (int a = 0; a < 3; ++a)
        {
            out.body.r[a] = s.q.r[a];
            out.body.v[a] = s.q.v[a];
            out.body.w[a] = s.q.w[a];
        }
        for (int k = 0; k < 9; ++k) out.body.R[k] = s.q.R[k];
        out.t = s.q.t;
        out.dt_current = s.dt_current;
        out.last_gap = s.last_gap;
        out.last_penetration = s.last_pen;
        out.last_normal_velocity = s.last_vn;
        out.last_toi = s.last_toi;
        out.phase = s.phase;
        out.stable_count = s.stable_count;
        out.release_count = s.release_count;
        out.min_dt_hits = s.min_dt_hits;
        if (h_out) h_out[sc] = h;
        if (unfinished && s.q.t < t_end[sc] - 1e-15) atomicAdd(unfinished, 1);
        if (b.stats)
        {
            atomicAdd(b.stats, (unsigned long long)s.n_newton);
            atomicAdd(b.stats + 1, (unsigned long long)s.n_resid);
            atomicAdd(b.stats + 2, (unsigned long long)s.n_solves);
        }
    }
}

} // namespace
} // namespace sdfo

// The arguments a captured run of integrate-mode launches was recorded with.
struct BeGraphKey
{
    void* scenes = nullptr;
    int64_t n = -1;
    const double* t_end = nullptr;
    double dt = 0.0;
    int launches = 0;
    int* unfinished = nullptr;
    int threads = 0;
    bool operator==(const BeGraphKey& o) const
    {
        return scenes == o.scenes && n == o.n && t_end == o.t_end && dt == o.dt && launches == o.launches &&
               unfinished == o.unfinished && threads == o.threads;
    }
};

struct sdfo_be_stepper
{
    const sdfo_contact_pair* pair = nullptr;
    sdfo::BeView view{};
    int64_t capacity = 0;
    int threads = 256;
    // integrate mode: the last captured graph, the stream it was captured
    // on, and the unfinished-scene counter (device) with its pinned mirror
    BeGraphKey key{};
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capture = nullptr;
    int* d_unfinished = nullptr;
    int* h_unfinished = nullptr;
    ~sdfo_be_stepper()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (capture) cudaStreamDestroy(capture);
        if (h_unfinished) cudaFreeHost(h_unfinished);
        sdfo::device_free(d_unfinished);
        sdfo::device_free(view.cg);
        sdfo::device_free(view.cgrad);
        sdfo::device_free(view.cvalid);
        sdfo::device_free(view.stats);
    }
};

namespace sdfo {
namespace {

void launch_step(const sdfo_be_stepper* st, sdfo_be_scene* scenes, int64_t n, const double* dt, double* h,
                 const double* t_end, double dt_max, int* unfinished, cudaStream_t s)
{
#define SDFO_BE_LAUNCH(EX)                                                                                  \
    if (st->threads == 32)                                                                                  \
        k_be_step<256, true, EX><<<(unsigned)((n + 7) / 8), 256, EX ? jac_smem_bytes<256>() : 0, s>>>(     \
            st->view, scenes, (int)n, dt, h, t_end, dt_max, unfinished);                                    \
    else if (st->threads == 128)                                                                            \
        k_be_step<128, false, EX><<<(unsigned)n, 128, EX ? jac_smem_bytes<128>() : 0, s>>>(                 \
            st->view, scenes, (int)n, dt, h, t_end, dt_max, unfinished);                                    \
    else                                                                                                    \
        k_be_step<256, false, EX><<<(unsigned)n, 256, EX ? jac_smem_bytes<256>() : 0, s>>>(                 \
            st->view, scenes, (int)n, dt, h, t_end, dt_max, unfinished);
    if (st->view.p.tangent == SDFO_BE_TANGENT_EXACT)
    {
        SDFO_BE_LAUNCH(true)
    }
    else
    {
        SDFO_BE_LAUNCH(false)
    }
#undef SDFO_BE_LAUNCH
    SDFO_CHECK_LAUNCH();
}

// Records `k.launches` integrate-mode launches (the counter cleared first,
// the last launch counting the scenes still short of t_end) as one graph.
cudaGraphExec_t capture_advance(sdfo_be_stepper* st, const BeGraphKey& k)
{
    if (!st->capture) SDFO_CUDA(cudaStreamCreateWithFlags(&st->capture, cudaStreamNonBlocking));
    cudaStream_t cs = st->capture;
    SDFO_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try
    {
        if (k.unfinished) SDFO_CUDA(cudaMemsetAsync(k.unfinished, 0, sizeof(int), cs));
        for (int i = 0; i < k.launches; ++i)
            launch_step(st, static_cast<sdfo_be_scene*>(k.scenes), k.n, nullptr, nullptr, k.t_end, k.dt,
                        i + 1 == k.launches ? k.unfinished : nullptr, cs);
    }
    catch (...)
    {
        cudaStreamEndCapture(cs, &graph);
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        throw;
    }
    SDFO_CUDA(cudaStreamEndCapture(cs, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    SDFO_CUDA(e);
    return exec;
}

void advance(sdfo_be_stepper* st, sdfo_be_scene* scenes, int64_t n, const double* t_end, double dt, int launches,
             int* unfinished, cudaStream_t s)
{
    BeGraphKey k;
    k.scenes = scenes;
    k.n = n;
    k.t_end = t_end;
    k.dt = dt;
    k.launches = launches;
    k.unfinished = unfinished;
    k.threads = st->threads;
    if (!st->exec || !(st->key == k))
    {
        if (st->exec)
        {
            cudaGraphExecDestroy(st->exec);
            st->exec = nullptr;
        }
        st->exec = capture_advance(st, k);
        st->key = k;
    }
    SDFO_CUDA(cudaGraphLaunch(st->exec, s));
}

} // namespace
} // namespace sdfo

using namespace sdfo;

extern "C" {

void sdfo_be_params_default(sdfo_be_params* p)
{
    if (!p) return;
    p->max_iter = 20;
    p->line_search = 1;
    p->max_toi_bisect_iter = 60;
    p->stable_steps = 5;
    p->release_steps = 3;
    p->tangent = SDFO_BE_TANGENT_REFERENCE;
    p->tol = 1e-8;
    p->pen_max = 1e-6;
    p->dt_min = 1e-8;
    p->dt_impact = 1e-7;
    p->dt_contact = 1e-5;
    p->dt_max_contact = 1e-4;
    p->dt_normal = 1e-3;
    p->dt_growth = 1.5;
}

void sdfo_be_scene_init(sdfo_be_scene* s, const sdfo_body_state* body, double t, const sdfo_be_params* p)
{
    if (!s) return;
    std::memset(s, 0, sizeof(*s));
    if (body) s->body = *body;
    s->t = t;
    s->dt_current = p ? p->dt_normal : 1e-3;
    s->last_gap = INFINITY;
    s->last_toi = INFINITY;
    s->phase = 0;
}

int sdfo_be_stepper_create(const sdfo_contact_pair* pair, const sdfo_contact_params* contact,
                           const sdfo_rigid_body* body_a, const sdfo_body_state* body_b,
                           const sdfo_be_params* params, int64_t max_scenes, sdfo_be_stepper** out)
{
    return guarded([&] {
        SDFO_REQUIRE(pair && contact && body_a && body_b && params && out, SDFO_ERR_INVALID_ARGUMENT,
                     "NULL argument");
        *out = nullptr;
        SDFO_REQUIRE(pair->grid != nullptr, SDFO_ERR_INVALID_ARGUMENT, "pair was created without a grid");
        const sdfo_grid* g = pair->grid;
        SDFO_REQUIRE(g->info.layout == SDFO_LAYOUT_DENSE && g->d.phi64 != nullptr, SDFO_ERR_UNSUPPORTED,
                     "BE stepping samples a dense grid's FP64 values (build, load or create it from FP64 data)");
        SDFO_REQUIRE(max_scenes > 0 && max_scenes <= 0x7fffffff, SDFO_ERR_INVALID_ARGUMENT, "bad scene count");
        SDFO_REQUIRE(params->max_iter >= 0 && params->max_toi_bisect_iter >= 0, SDFO_ERR_INVALID_ARGUMENT,
                     "negative iteration count");
        SDFO_REQUIRE(body_a->mass > 0.0, SDFO_ERR_INVALID_ARGUMENT, "body mass must be positive");
        SDFO_REQUIRE(params->tangent == SDFO_BE_TANGENT_REFERENCE || params->tangent == SDFO_BE_TANGENT_EXACT,
                     SDFO_ERR_INVALID_ARGUMENT, "unknown tangent mode");
        std::unique_ptr<sdfo_be_stepper> st(new sdfo_be_stepper());
        st->pair = pair;
        BeView& b = st->view;
        b.g = make_view(g);
        b.phi64 = g->d.phi64;
        b.nq = (int)pair->nq;
        b.nleaves = pair->nleaves;
        b.cull = pair->narrow_margin >= 0.0 ? 1 : 0;
        b.px = pair->px64;
        b.pw = pair->pw64;
        b.pleaf = pair->pleaf;
        b.ox = pair->ox64;
        b.ow = pair->ow64;
        b.leaf_box = pair->leaf_box;
        for (int a = 0; a < 6; ++a) b.root[a] = pair->root[a];
        for (int a = 0; a < 3; ++a)
        {
            b.bmin[a] = g->info.bmin[a];
            b.bmax[a] = g->info.bmax[a];
            b.rB[a] = body_b->r[a];
            b.vB[a] = body_b->v[a];
            b.wB[a] = body_b->w[a];
            b.gravity[a] = body_a->gravity[a];
        }
        for (int k = 0; k < 9; ++k)
        {
            b.RB[k] = body_b->R[k];
            b.Ib[k] = body_a->inertia[k];
        }
        b.box_margin = std::max(pair->narrow_margin, 0.05);
        b.narrow = pair->narrow_margin;
        b.mass = body_a->mass;
        // np.sum of the pair's (normalised) weights: the tangent's `area`
        double area = 0.0;
        if (pair->nq > 0)
        {
            std::vector<double> w((size_t)pair->nq);
            SDFO_CUDA(cudaMemcpy(w.data(), pair->ow64, sizeof(double) * pair->nq, cudaMemcpyDeviceToHost));
            for (double x : w) area += x;
        }
        b.area = area;
        b.c = *contact;
        b.p = *params;
        st->capacity = max_scenes;
        const size_t slots = (size_t)max_scenes * (size_t)std::max<int64_t>(pair->nq, 1);
        b.cg = dalloc<double>(slots);
        b.cgrad = dalloc<double>(3 * slots);
        b.cvalid = dalloc<unsigned char>(slots);
        if (params->tangent == SDFO_BE_TANGENT_EXACT)
        {
            // static + dynamic shared memory above 48 KB needs the opt-in
            SDFO_CUDA(cudaFuncSetAttribute(k_be_step<256, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           jac_smem_bytes<256>()));
            SDFO_CUDA(cudaFuncSetAttribute(k_be_step<256, false, true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, jac_smem_bytes<256>()));
            SDFO_CUDA(cudaFuncSetAttribute(k_be_step<128, false, true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, jac_smem_bytes<128>()));
        }
        b.stats = dalloc<unsigned long long>(3);
        SDFO_CUDA(cudaMemset(b.stats, 0, 3 * sizeof(unsigned long long)));
        *out = st.release();
    });
}

int sdfo_be_stepper_step(sdfo_be_stepper* st, sdfo_be_scene* d_scenes, int64_t n, const double* d_dt,
                         double* d_h, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(st != nullptr, SDFO_ERR_INVALID_ARGUMENT, "stepper is NULL");
        SDFO_REQUIRE(n >= 0 && n <= st->capacity, SDFO_ERR_INVALID_ARGUMENT,
                     "scene count exceeds the stepper's capacity");
        if (n == 0) return;
        SDFO_REQUIRE(d_scenes && d_dt, SDFO_ERR_INVALID_ARGUMENT, "scenes and step sizes are required");
        launch_step(st, d_scenes, n, d_dt, d_h, nullptr, 0.0, nullptr, as_stream(stream));
    });
}

int sdfo_be_stepper_advance(sdfo_be_stepper* st, sdfo_be_scene* d_scenes, int64_t n, const double* d_t_end,
                            double dt, int32_t launches, int32_t* d_unfinished, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(st != nullptr, SDFO_ERR_INVALID_ARGUMENT, "stepper is NULL");
        SDFO_REQUIRE(n >= 0 && n <= st->capacity, SDFO_ERR_INVALID_ARGUMENT,
                     "scene count exceeds the stepper's capacity");
        SDFO_REQUIRE(dt > 0.0, SDFO_ERR_INVALID_ARGUMENT, "dt must be positive");
        SDFO_REQUIRE(launches >= 1 && launches <= 4096, SDFO_ERR_INVALID_ARGUMENT,
                     "launches must be in [1, 4096]");
        cudaStream_t s = as_stream(stream);
        if (n == 0)
        {
            if (d_unfinished) SDFO_CUDA(cudaMemsetAsync(d_unfinished, 0, sizeof(int32_t), s));
            return;
        }
        SDFO_REQUIRE(d_scenes && d_t_end, SDFO_ERR_INVALID_ARGUMENT, "scenes and end times are required");
        advance(st, d_scenes, n, d_t_end, dt, launches, d_unfinished, s);
    });
}

int sdfo_be_stepper_integrate(sdfo_be_stepper* st, sdfo_be_scene* d_scenes, int64_t n, const double* d_t_end,
                              double dt, int32_t launches_per_check, int64_t max_launches, int64_t* launches_out,
                              int32_t* unfinished_out, void* stream)
{
    return guarded([&] {
        SDFO_REQUIRE(st != nullptr, SDFO_ERR_INVALID_ARGUMENT, "stepper is NULL");
        SDFO_REQUIRE(n >= 0 && n <= st->capacity, SDFO_ERR_INVALID_ARGUMENT,
                     "scene count exceeds the stepper's capacity");
        SDFO_REQUIRE(dt > 0.0, SDFO_ERR_INVALID_ARGUMENT, "dt must be positive");
        SDFO_REQUIRE(launches_per_check >= 1 && launches_per_check <= 4096, SDFO_ERR_INVALID_ARGUMENT,
                     "launches_per_check must be in [1, 4096]");
        SDFO_REQUIRE(max_launches >= 1, SDFO_ERR_INVALID_ARGUMENT, "max_launches must be positive");
        if (launches_out) *launches_out = 0;
        if (unfinished_out) *unfinished_out = 0;
        if (n == 0) return;
        SDFO_REQUIRE(d_scenes && d_t_end, SDFO_ERR_INVALID_ARGUMENT, "scenes and end times are required");
        if (!st->d_unfinished) st->d_unfinished = dalloc<int>(1);
        if (!st->h_unfinished) SDFO_CUDA(cudaHostAlloc(&st->h_unfinished, sizeof(int), cudaHostAllocDefault));
        cudaStream_t s = as_stream(stream);
        int64_t made = 0;
        while (made < max_launches)
        {
            advance(st, d_scenes, n, d_t_end, dt, launches_per_check, st->d_unfinished, s);
            made += launches_per_check;
            SDFO_CUDA(cudaMemcpyAsync(st->h_unfinished, st->d_unfinished, sizeof(int), cudaMemcpyDeviceToHost, s));
            SDFO_CUDA(cudaStreamSynchronize(s));
            if (*st->h_unfinished == 0) break;
        }
        if (launches_out) *launches_out = made;
        if (unfinished_out) *unfinished_out = *st->h_unfinished;
    });
}

int sdfo_be_stepper_set_threads(sdfo_be_stepper* st, int32_t threads)
{
    return guarded([&] {
        SDFO_REQUIRE(st != nullptr, SDFO_ERR_INVALID_ARGUMENT, "stepper is NULL");
        SDFO_REQUIRE(threads == 32 || threads == 128 || threads == 256, SDFO_ERR_INVALID_ARGUMENT,
                     "threads per scene must be 32, 128 or 256");
        st->threads = threads;
    });
}

int sdfo_be_stepper_stats(sdfo_be_stepper* st, uint64_t* out, int32_t reset)
{
    return guarded([&] {
        SDFO_REQUIRE(st != nullptr && out != nullptr, SDFO_ERR_INVALID_ARGUMENT, "NULL argument");
        unsigned long long v[3] = {0, 0, 0};
        SDFO_CUDA(cudaDeviceSynchronize());
        SDFO_CUDA(cudaMemcpy(v, st->view.stats, sizeof(v), cudaMemcpyDeviceToHost));
        for (int k = 0; k < 3; ++k) out[k] = (uint64_t)v[k];
        if (reset) SDFO_CUDA(cudaMemset(st->view.stats, 0, sizeof(v)));
    });
}

int sdfo_be_stepper_destroy(sdfo_be_stepper* st)
{
    delete st;
    return SDFO_OK;
}

} // extern "C"
