// ContactAware queries on grids with surface-feature candidates: the
// ContactAware branch of SdfOracle::queryFast (SdfOracle.cpp:296-423) and
// contactAwareQuery (SdfOracle.cpp:853-914).  One thread per point:
// nearest voxel (GridSpec::indexFromWorld), then for each of the voxel's
// candidates (at most 8) the normalised normal, the linear extrapolation
// gap = phi + n.(p - centre) and the witness p - gap n; the candidate with the
// smallest |gap| (first on ties) is the result.  A voxel without candidates
// answers with the FirstOrder query, as in the reference.
//
// Compiled with -fmad=false: the FP64 candidate arithmetic keeps the
// reference's operation order, so the selected candidate and every gap are
// the reference's values before the FP32 outputs round them.
#include <algorithm>
#include <cfloat>
#include <mutex>

#include "interp.cuh"

namespace sdfo {
namespace {

constexpr int kThreads = 256;

template <typename PT>
__device__ __forceinline__ void load_pt(const PT* pts, int64_t q, double p[3])
{
    p[0] = (double)__ldcs(pts + 3 * q);
    p[1] = (double)__ldcs(pts + 3 * q + 1);
    p[2] = (double)__ldcs(pts + 3 * q + 2);
}

// The ContactAware answer for point p, query q.
template <bool SPARSE, int BD>
__device__ __forceinline__ void ca_query_one(const GridView& g, const double p[3], int64_t q,
                                             const QueryOutputs& o, const CandidateOutputs& co)
{
    // indexFromWorld (GridSpec.h:37-45) and the in-grid / stored-block test
    int ijk[3];
    bool inb = true;
    const int nn[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        const double f = frac_coord_fast<true>(p[a], g.bmin[a], g.voxel[a], g.ivoxel[a]);
        if (!(f > -1.0 && f < (double)nn[a] + 1.0))
        {
            inb = false;
            ijk[a] = 0;
            continue;
        }
        ijk[a] = (int)round(f);
        inb = inb && ijk[a] >= 0 && ijk[a] < nn[a];
    }
    int64_t v = -1;
    if (inb) v = SPARSE ? sparse_index<BD>(g, ijk[0], ijk[1], ijk[2]) : dense_index(g, ijk[0], ijk[1], ijk[2]);
    double gap = 0.0, nrm[3] = {1.0, 0.0, 0.0}, wit[3] = {0.0, 0.0, 0.0};
    int ncand = 0;
    const int cnt = v >= 0 ? min((int)__ldg(g.ca_count + v), g.ca_stride) : 0;
    if (v >= 0 && cnt <= 0)
    {
        // no candidate at this voxel: FirstOrder (SdfOracle.cpp:329, 385)
        Interp r;
        float unit[3];
        evaluate<SDFO_FIRST_ORDER, SPARSE, BD, false>(g, p, r, unit);
        gap = r.gap;
        for (int a = 0; a < 3; ++a)
        {
            nrm[a] = unit[a];
            wit[a] = p[a] - gap * nrm[a];
        }
        ncand = 1;
        if (co.kgap)
        {
            co.kgap[8 * q] = (float)gap;
            co.kbranch[8 * q] = 0;
            for (int a = 0; a < 3; ++a)
            {
                co.knormal[24 * q + a] = (float)nrm[a];
                co.kwitness[24 * q + a] = (float)wit[a];
            }
        }
    }
    else if (v >= 0)
    {
        const double c[3] = {g.bmin[0] + g.voxel[0] * (ijk[0] + 0.5),
                             g.bmin[1] + g.voxel[1] * (ijk[1] + 0.5),
                             g.bmin[2] + g.voxel[2] * (ijk[2] + 0.5)};
        const double dx[3] = {p[0] - c[0], p[1] - c[1], p[2] - c[2]};
        ncand = cnt < 8 ? cnt : 8;
        double best = DBL_MAX;
        for (int k = 0; k < ncand; ++k)
        {
            const int64_t idx = v * g.ca_stride + k;
            double m[3];
            double phi;
            if (SPARSE)
            {
                phi = (double)__ldg(g.ca_phi32 + idx);
                for (int a = 0; a < 3; ++a) m[a] = (double)__ldg(g.ca_n32 + 3 * idx + a);
            }
            else
            {
                phi = __ldg(g.ca_phi64 + idx);
                for (int a = 0; a < 3; ++a) m[a] = __ldg(g.ca_n64 + 3 * idx + a);
            }
            const double l = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            if (l > 1.0e-15)
            {
                for (int a = 0; a < 3; ++a) m[a] = m[a] / l;
            }
            else
            {
                m[0] = 1.0;
                m[1] = m[2] = 0.0;
            }
            const double gk = phi + (m[0] * dx[0] + m[1] * dx[1] + m[2] * dx[2]);
            const double wk[3] = {p[0] - gk * m[0], p[1] - gk * m[1], p[2] - gk * m[2]};
            if (co.kgap)
            {
                co.kgap[8 * q + k] = (float)gk;
                co.kbranch[8 * q + k] = __ldg(g.ca_branch + idx);
                for (int a = 0; a < 3; ++a)
                {
                    co.knormal[24 * q + 3 * k + a] = (float)m[a];
                    co.kwitness[24 * q + 3 * k + a] = (float)wk[a];
                }
            }
            if (fabs(gk) < best)
            {
                best = fabs(gk);
                gap = gk;
                for (int a = 0; a < 3; ++a)
                {
                    nrm[a] = m[a];
                    wit[a] = wk[a];
                }
            }
        }
    }
    if (co.kgap)
    {
        co.ncand[q] = ncand;
        for (int k = ncand; k < 8; ++k)
        {
            co.kgap[8 * q + k] = 0.f;
            co.kbranch[8 * q + k] = -1;
            for (int a = 0; a < 3; ++a)
            {
                co.knormal[24 * q + 3 * k + a] = a == 0 ? 1.f : 0.f;
                co.kwitness[24 * q + 3 * k + a] = 0.f;
            }
        }
    }
    __stcs(o.gap + q, (float)gap);
    if (o.valid) o.valid[q] = v >= 0 ? 1 : 0;
    for (int a = 0; a < 3; ++a)
    {
        if (o.grad) __stcs(o.grad + 3 * q + a, (float)nrm[a]);
        if (o.unit) __stcs(o.unit + 3 * q + a, (float)nrm[a]);
        if (o.witness) __stcs(o.witness + 3 * q + a, (float)wit[a]);
    }
}

template <bool SPARSE, int BD, typename PT>
__global__ void __launch_bounds__(kThreads)
    k_query_ca(GridView g, const PT* __restrict__ pts, int64_t n, QueryOutputs o, CandidateOutputs co)
{
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= n) return;
    double p[3];
    load_pt(pts, q, p);
    ca_query_one<SPARSE, BD>(g, p, q, o, co);
}

// Persistent variant for FP32 points on sparse grids
// (sdfo_tuning.query_walk): CTA c walks the contiguous tile range
// [ntiles c / G, ntiles (c + 1) / G) of kThreads queries and each thread
// loads its next point before it answers the current one, so the point load
// leaves the chain point -> brick -> voxel -> candidates.
template <bool SPARSE, int BD>
__global__ void __launch_bounds__(kThreads)
    k_query_ca_walk(GridView g, const float* __restrict__ pts, int64_t n, QueryOutputs o, CandidateOutputs co)
{
    const int64_t ntiles = (n + kThreads - 1) / kThreads;
    const int64_t t_begin = ntiles * blockIdx.x / gridDim.x;
    const int64_t t_end = ntiles * (blockIdx.x + 1) / gridDim.x;
    int64_t q = t_begin * kThreads + threadIdx.x;
    float xn[3] = {0.f, 0.f, 0.f};
    if (t_begin < t_end && q < n)
        for (int a = 0; a < 3; ++a) xn[a] = __ldcs(pts + 3 * q + a);
    for (int64_t t = t_begin; t < t_end; ++t)
    {
        const int64_t qc = q;
        const double p[3] = {xn[0], xn[1], xn[2]};
        q += kThreads;
        if (t + 1 < t_end && q < n)
            for (int a = 0; a < 3; ++a) xn[a] = __ldcs(pts + 3 * q + a);
        if (qc < n) ca_query_one<SPARSE, BD>(g, p, qc, o, co);
    }
}

// One candidate per valid point from a query's own result (fastFromQueryResult,
// SdfOracle.cpp:86-120).
__global__ void k_single_candidate(int64_t n, const float* __restrict__ gap,
                                   const float* __restrict__ unit, const float* __restrict__ wit,
                                   const uint8_t* __restrict__ valid, CandidateOutputs co)
{
    const int64_t q = (int64_t)blockIdx.x * kThreads + threadIdx.x;
    if (q >= n) return;
    const bool ok = valid[q] != 0;
    co.ncand[q] = ok ? 1 : 0;
    for (int k = 0; k < 8; ++k)
    {
        const bool first = ok && k == 0;
        co.kgap[8 * q + k] = first ? gap[q] : 0.f;
        co.kbranch[8 * q + k] = first ? 0 : -1;
        for (int a = 0; a < 3; ++a)
        {
            co.knormal[24 * q + 3 * k + a] = first ? unit[3 * q + a] : (a == 0 ? 1.f : 0.f);
            co.kwitness[24 * q + 3 * k + a] = first ? wit[3 * q + a] : 0.f;
        }
    }
}

template <bool SPARSE, int BD>
void launch_ca2(const GridView& v, const void* pts, bool f64, int64_t n, const QueryOutputs& o,
                const CandidateOutputs& co, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
    // sparse grids only: measured on the hollow cylinder's candidate grids
    // (1M points), the walk took sparse queries from 10.2 to 11.6 G/s but
    // dense ones (FP64 candidates, 4 per voxel) from 13.5 down to 10.4 (10.7
    // in grid-stride order): there the work per query varies (voxels without
    // candidates answer with a FirstOrder query), which fresh CTAs balance
    // and a fixed persistent assignment does not
    if (SPARSE && !f64 && query_walk())
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
                SDFO_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_query_ca_walk<SPARSE, BD>, kThreads, 0));
                per_sm[dev & 63] = r > 0 ? r : 1;
            }
            b = per_sm[dev & 63];
        }
        const unsigned g = (unsigned)std::min<int64_t>(blocks, (int64_t)current_sm_count() * b);
        k_query_ca_walk<SPARSE, BD><<<g, kThreads, 0, s>>>(v, static_cast<const float*>(pts), n, o, co);
    }
    else if (f64)
        k_query_ca<SPARSE, BD, double><<<blocks, kThreads, 0, s>>>(v, static_cast<const double*>(pts), n, o, co);
    else
        k_query_ca<SPARSE, BD, float><<<blocks, kThreads, 0, s>>>(v, static_cast<const float*>(pts), n, o, co);
}

} // namespace

void launch_query_ca(const GridView& v, const void* pts, bool f64, int64_t n, const QueryOutputs& o,
                     const CandidateOutputs& co, cudaStream_t s)
{
    if (n <= 0) return;
    if (v.layout == SDFO_LAYOUT_DENSE)
        launch_ca2<false, 0>(v, pts, f64, n, o, co, s);
    else if (v.bd == 8)
        launch_ca2<true, 8>(v, pts, f64, n, o, co, s);
    else
        launch_ca2<true, 0>(v, pts, f64, n, o, co, s);
    SDFO_CHECK_LAUNCH();
}

void launch_single_candidate(int64_t n, const float* gap, const float* unit, const float* wit,
                             const uint8_t* valid, const CandidateOutputs& co, cudaStream_t s)
{
    if (n <= 0) return;
    k_single_candidate<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(n, gap, unit, wit,
                                                                                     valid, co);
    SDFO_CHECK_LAUNCH();
}

} // namespace sdfo
