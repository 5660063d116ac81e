// Device-side grid addressing and interpolants shared by the query, backward
// and contact kernels.
//
// Interpolants restate the reference's SdfOracle query modes:
//   trilinear  - SdfOracle.cpp:524-596 (8-corner lerp of phi, analytic gradient)
//   tricubic   - SdfOracle.cpp:932-1092 (tensor cubic Hermite over the 8 cell
//                corners with values phi and slopes n*h; no cross terms)
//   first/second order - SdfOracle.cpp:448-520 (Taylor at the nearest voxel)
// Arithmetic is FP32 (storage is FP32/FP16); the cell index and fractional
// coordinate are computed in FP64 exactly as the reference does,
// f = (p - bmin) / voxel - 0.5, so every query selects the reference's cell.
#pragma once

#include "sdfo_internal.cuh"

namespace sdfo {

struct Cell
{
    int i0, j0, k0;  // lower corner (trilinear/tricubic) or nearest voxel
    float u, v, w;   // fractional position in the cell
    bool ok;         // inside the index domain
};

// Fractional grid coordinate as in GridSpec/trilinearQuery,
// f = (p - bmin).cwiseQuotient(voxel) - 0.5, without the FP64 division where that cannot change
// the cell where it cannot change the result: (p - bmin) * (1/voxel) is within 2^-39 of the quotient for
// |f| < 2^12, so when it lies more than 2^-30 from the decision points
// (integers for the cell index, half-integers for the nearest voxel) both
// select the same cell, and the fraction differs by < 2^-39 (below FP32
// resolution); near a decision point the reference's division is used.
template <bool NEAREST>
__device__ __forceinline__ double frac_coord_fast(double p, double bmin, double voxel,
                                                  double ivoxel)
{
    const double d = p - bmin;
    const double f = d * ivoxel - 0.5;
    const double t = NEAREST ? f + 0.5 : f;
    const double fr = t - floor(t);
    if (fr > 0x1p-30 && fr < 1.0 - 0x1p-30 && fabs(f) < 4096.0) return f;
    return d / voxel - 0.5;
}

// Lower-corner cell of p; ok iff i0 >= 0 and i0 + 1 < n on every axis.
__device__ __forceinline__ Cell cell_of(const GridView& g, const double p[3])
{
    Cell c;
    double f[3];
    int lo[3];
    bool ok = true;
    const int n[3] = {g.nx, g.ny, g.nz};
    float fr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        f[a] = frac_coord_fast<false>(p[a], g.bmin[a], g.voxel[a], g.ivoxel[a]);
        // NaN / huge coordinates are outside the domain.
        if (!(f[a] >= -1.0 && f[a] < (double)n[a]))
        {
            ok = false;
            lo[a] = 0;
            fr[a] = 0.f;
            continue;
        }
        const double fl = floor(f[a]);
        lo[a] = (int)fl;
        fr[a] = (float)(f[a] - fl);
        ok = ok && lo[a] >= 0 && lo[a] + 1 < n[a];
    }
    c.i0 = lo[0];
    c.j0 = lo[1];
    c.k0 = lo[2];
    c.u = fr[0];
    c.v = fr[1];
    c.w = fr[2];
    c.ok = ok;
    return c;
}

// Nearest voxel (GridSpec::indexFromWorld, GridSpec.h:37-45) with its
// in-bounds flag; dx = p - centre (FP64 then FP32).
__device__ __forceinline__ bool nearest_voxel(const GridView& g, const double p[3], int ijk[3],
                                              float dx[3])
{
    const int n[3] = {g.nx, g.ny, g.nz};
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
        const double f = frac_coord_fast<true>(p[a], g.bmin[a], g.voxel[a], g.ivoxel[a]);
        if (!(f > -1.0 && f < (double)n[a] + 1.0))
        {
            ok = false;
            ijk[a] = 0;
            dx[a] = 0.f;
            continue;
        }
        ijk[a] = (int)round(f);
        ok = ok && ijk[a] >= 0 && ijk[a] < n[a];
        const double c = g.bmin[a] + g.voxel[a] * (ijk[a] + 0.5);
        dx[a] = (float)(p[a] - c);
    }
    return ok;
}

// One 256-bit read-only load (sm_100: ld.global.nc.v8.f32) of a 32-byte
// aligned record: a single L1 request and one 32-byte sector.
__device__ __forceinline__ void ld256(const float4* p, float4& a, float4& b)
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

__device__ __forceinline__ int64_t dense_index(const GridView& g, int i, int j, int k)
{
    return (int64_t)i + (int64_t)g.nx * ((int64_t)j + (int64_t)g.ny * (int64_t)k);
}

// Stored-voxel index of (i,j,k) in a sparse grid or -1 when its block is not
// stored (SparseSdfData::blockForVoxel + sampleFromBlock, SdfData.h:224-302).
// BD = block_dim when known at compile time, 0 for the runtime value.
template <int BD>
__device__ __forceinline__ int64_t sparse_index(const GridView& g, int i, int j, int k)
{
    const int bd = BD > 0 ? BD : g.bd;
    const int bi = i / bd, bj = j / bd, bk = k / bd;
    const int slot = __ldg(g.table + bi + g.nbx * (bj + g.nby * bk));
    if (slot < 0) return -1;
    const int local = (i - bi * bd) + bd * ((j - bj * bd) + bd * (k - bk * bd));
    return (int64_t)slot * (bd * bd * bd) + local;
}

// FP16 payload: {phi_q, nx, ny, nz} halves; phi = phi_q * scale + offset.
__device__ __forceinline__ float4 decode_fp16(ushort4 q, float2 aff)
{
    float4 r;
    r.x = __half2float(__ushort_as_half(q.x)) * aff.x + aff.y;
    r.y = __half2float(__ushort_as_half(q.y));
    r.z = __half2float(__ushort_as_half(q.z));
    r.w = __half2float(__ushort_as_half(q.w));
    return r;
}

template <int BD>
__device__ __forceinline__ float4 load_stored(const GridView& g, int64_t idx)
{
    if (g.storage == SDFO_STORAGE_FP16)
    {
        const int V = (BD > 0 ? BD : g.bd);
        const int64_t brick = idx / (V * V * V);
        return decode_fp16(__ldg(g.phin16 + idx), __ldg(g.brick_affine + brick));
    }
    return __ldg(g.phin + idx);
}

// Gathers the 8 cell corners (corner c = di + 2 dj + 4 dk) as {phi, n}.
// Returns false when a sparse corner's block is missing.
template <bool SPARSE, int BD>
__device__ __forceinline__ bool gather_corners(const GridView& g, const Cell& c, float4 out[8],
                                               int64_t idx[8])
{
    if (!SPARSE)
    {
        const int64_t base = dense_index(g, c.i0, c.j0, c.k0);
        const int64_t sx = 1, sy = g.nx, sz = (int64_t)g.nx * g.ny;
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            idx[q] = base + ((q & 1) ? sx : 0) + ((q & 2) ? sy : 0) + ((q & 4) ? sz : 0);
            out[q] = __ldg(g.phin + idx[q]);
        }
        return true;
    }
    const int bd = BD > 0 ? BD : g.bd;
    const int bi = c.i0 / bd, bj = c.j0 / bd, bk = c.k0 / bd;
    const int li = c.i0 - bi * bd, lj = c.j0 - bj * bd, lk = c.k0 - bk * bd;
    bool ok = true;
    if (li < bd - 1 && lj < bd - 1 && lk < bd - 1)
    {
        // the whole cell lies in one brick (343 of 512 cells for 8^3):
        // one table lookup
        const int slot = __ldg(g.table + bi + g.nbx * (bj + g.nby * bk));
        if (slot < 0) return false;
        const int64_t i0 = (int64_t)slot * (bd * bd * bd) + li + bd * (lj + bd * lk);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            idx[q] = i0 + ((q & 1) ? 1 : 0) + ((q & 2) ? bd : 0) + ((q & 4) ? bd * bd : 0);
    }
    else
    {
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            idx[q] = sparse_index<BD>(g, c.i0 + (q & 1), c.j0 + ((q >> 1) & 1), c.k0 + (q >> 2));
            ok = ok && idx[q] >= 0;
        }
    }
    if (!ok) return false;
#pragma unroll
    for (int q = 0; q < 8; ++q) out[q] = load_stored<BD>(g, idx[q]);
    return true;
}

// The 8 cell corners of a sparse 8^3-brick grid as rows: for each (dj, dk)
// the x-pair (i0, i0 + 1).  Each distinct brick the cell touches is looked
// up once (1.42 lookups per uniformly placed cell, instead of one per corner
// when the cell crosses a brick face).  FP32 with the grid's x-pair records
// (GridView::xpair, 32 bytes per stored voxel): one 256-bit load per row;
// without them a pair starting on an even x is one 256-bit load, otherwise
// two 128-bit loads.  FP16: the 32-byte chunk
// of four voxels holding i0 is one 256-bit load; i0 mod 4 == 3 needs a second,
// 64-bit load for i0 + 1; the brick's affine phi map is read once per brick.
// Needs the pool on a 32-byte boundary (GridView::phin_a32).  Same values and
// validity as gather_corners.
// One FP16 voxel {phi, nx, ny, nz} held as two 32-bit words (low half
// first), decoded as decode_fp16 does.
__device__ __forceinline__ float4 decode_fp16_words(unsigned w0, unsigned w1, float2 aff)
{
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&w0));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&w1));
    return make_float4(a.x * aff.x + aff.y, a.y, b.x, b.y);
}

template <int ST = 0>
__device__ __forceinline__ bool gather_rows_b8(const GridView& g, const Cell& c, float4 out[8])
{
    constexpr int bd = 8, V = 512;
    const int bi = c.i0 >> 3, bj = c.j0 >> 3, bk = c.k0 >> 3;
    const int li = c.i0 & 7, lj = c.j0 & 7, lk = c.k0 & 7;
    const bool cx = li == 7, cy = lj == 7, cz = lk == 7;
    const int32_t* tb = g.table + bi + g.nbx * (bj + g.nby * bk);
    const int sy = g.nbx, sz = g.nbx * g.nby;
    // s[dz][dy][dx]: slots of the bricks the cell touches
    int s[2][2][2];
    s[0][0][0] = __ldg(tb);
    s[0][0][1] = cx ? __ldg(tb + 1) : s[0][0][0];
    s[0][1][0] = cy ? __ldg(tb + sy) : s[0][0][0];
    s[0][1][1] = cx ? (cy ? __ldg(tb + sy + 1) : s[0][0][1]) : s[0][1][0];
    s[1][0][0] = cz ? __ldg(tb + sz) : s[0][0][0];
    s[1][0][1] = cz ? (cx ? __ldg(tb + sz + 1) : s[1][0][0]) : s[0][0][1];
    s[1][1][0] = cz ? (cy ? __ldg(tb + sz + sy) : s[1][0][0]) : s[0][1][0];
    s[1][1][1] = cz ? (cx && cy ? __ldg(tb + sz + sy + 1) : (cx ? s[1][0][1] : s[1][1][0])) : s[0][1][1];
    if ((s[0][0][0] | s[0][0][1] | s[0][1][0] | s[0][1][1] | s[1][0][0] | s[1][0][1] | s[1][1][0] |
         s[1][1][1]) < 0)
        return false;
    // ST: the pool's storage when the caller knows it (1 FP32, 2 FP16), else 0
    const bool fp16 = ST == 2 || (ST == 0 && g.storage == SDFO_STORAGE_FP16);
    // FP16: the affine phi map of the cell's first brick, read once; rows in
    // other bricks (cells on a brick face) read theirs
    const float2 aff000 = fp16 ? __ldg(g.brick_affine + s[0][0][0]) : make_float2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
        const int dj = r & 1, dk = r >> 1;
        // the row's bricks (s[dk][dj] equals s[0][..] / s[..][0] when the
        // cell does not cross that face)
        const int ly = (lj + dj) & 7, lz = (lk + dk) & 7;
        const int s0 = s[dk][dj][0], s1 = s[dk][dj][1];
        const int64_t row0 = (int64_t)s0 * V + bd * (ly + bd * lz);
        float4& a = out[2 * r];
        float4& b = out[2 * r + 1];
        if (!fp16 && g.xpair)
        {
            // the row's pair record {v, v + x}, the +x voxel taken across the
            // brick face (validity from the table lookups above)
            ld256(g.xpair + 2 * (row0 + li), a, b);
        }
        else if (!fp16)
        {
            if ((li & 1) == 0)
                ld256(g.phin + row0 + li, a, b);
            else
            {
                a = __ldg(g.phin + row0 + li);
                b = __ldg(g.phin + (cx ? (int64_t)s1 * V + bd * (ly + bd * lz) : row0 + li + 1));
            }
        }
        else
        {
            // FP16 voxels of 8 bytes: li even, the pair in one aligned
            // 16-byte load (li + 1 is in the same brick); li odd, two 8-byte
            // loads, the second across the brick face when li == 7
            const float2 af0 = s0 == s[0][0][0] ? aff000 : __ldg(g.brick_affine + s0);
            const ushort4* r16 = g.phin16 + row0 + li;
            if ((li & 1) == 0)
            {
                const uint4 w = __ldg(reinterpret_cast<const uint4*>(r16));
                a = decode_fp16_words(w.x, w.y, af0);
                b = decode_fp16_words(w.z, w.w, af0);
            }
            else
            {
                a = decode_fp16(__ldg(r16), af0);
                const int64_t i1 = cx ? (int64_t)s1 * V + bd * (ly + bd * lz) : row0 + li + 1;
                const float2 af1 = s1 == s0 ? af0 : __ldg(g.brick_affine + s1);
                b = decode_fp16(__ldg(g.phin16 + i1), af1);
            }
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// cubic Hermite basis: h00, h10, h01, h11 and their first/second derivatives
// (SdfOracle.cpp:976-1012 for the values and first derivatives).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void hermite(float t, float b[4], float d[4])
{
    const float t2 = t * t;
    b[0] = t2 * (2.f * t - 3.f) + 1.f;
    b[1] = t * (t * (t - 2.f) + 1.f);
    b[2] = t2 * (3.f - 2.f * t);
    b[3] = t2 * (t - 1.f);
    d[0] = 6.f * t * (t - 1.f);
    d[1] = t * (3.f * t - 4.f) + 1.f;
    d[2] = 6.f * t * (1.f - t);
    d[3] = t * (3.f * t - 2.f);
}
__device__ __forceinline__ void hermite2(float t, float s[4])
{
    s[0] = 12.f * t - 6.f;
    s[1] = 6.f * t - 4.f;
    s[2] = 6.f - 12.f * t;
    s[3] = 6.f * t - 2.f;
}

// x-collapse of the tensor Hermite interpolant for each (dj,dk) corner pair:
// X0 = sum_di P0 phi + P1 gx,  Xy = sum_di P0 gy,  Xz = sum_di P0 gz.
struct XColl
{
    float x0[4], xy[4], xz[4];
};

__device__ __forceinline__ XColl collapse_x(const float bx[4], const float phi[8],
                                            const float gx[8], const float gy[8],
                                            const float gz[8])
{
    XColl r;
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        const int c0 = 2 * q, c1 = 2 * q + 1;
        r.x0[q] = bx[0] * phi[c0] + bx[1] * gx[c0] + bx[2] * phi[c1] + bx[3] * gx[c1];
        r.xy[q] = bx[0] * gy[c0] + bx[2] * gy[c1];
        r.xz[q] = bx[0] * gz[c0] + bx[2] * gz[c1];
    }
    return r;
}

// yz-collapse: sum_dk R0 (sum_dj Q0 X0 + Q1 Xy) + R1 (sum_dj Q0 Xz).
__device__ __forceinline__ float collapse_yz(const XColl& x, const float by[4], const float bz[4])
{
    float y0[2], yz[2];
#pragma unroll
    for (int dk = 0; dk < 2; ++dk)
    {
        const int q0 = 2 * dk, q1 = 2 * dk + 1;
        y0[dk] = by[0] * x.x0[q0] + by[1] * x.xy[q0] + by[2] * x.x0[q1] + by[3] * x.xy[q1];
        yz[dk] = by[0] * x.xz[q0] + by[2] * x.xz[q1];
    }
    return bz[0] * y0[0] + bz[1] * yz[0] + bz[2] * y0[1] + bz[3] * yz[1];
}

struct Interp
{
    float gap;
    float g[3];   // raw gradient
    float H[6];   // xx, xy, xz, yy, yz, zz
};

// Tricubic Hermite (SdfOracle.cpp:932-1092) over corners {phi, n}; slopes
// n * h; gradient = d/du / h; optional Hessian.  The value weights sum to 1
// and every derivative's weights sum to 0, so phi is interpolated relative to
// corner 0 (phi_c - phi_0) and phi_0 added back to the value only: the FP32
// derivative sums then carry errors of order ulp(h), not ulp(|phi|).
template <bool HESS>
__device__ __forceinline__ Interp tricubic(const float4 c[8], float u, float v, float w,
                                           const float h[3], const float ih[3])
{
    float phi[8], gx[8], gy[8], gz[8];
    const float phi0 = c[0].x;
#pragma unroll
    for (int q = 0; q < 8; ++q)
    {
        phi[q] = c[q].x - phi0;
        gx[q] = c[q].y * h[0];
        gy[q] = c[q].z * h[1];
        gz[q] = c[q].w * h[2];
    }
    float bx[4], dx[4], by[4], dy[4], bz[4], dz[4];
    hermite(u, bx, dx);
    hermite(v, by, dy);
    hermite(w, bz, dz);
    const XColl xa = collapse_x(bx, phi, gx, gy, gz);
    const XColl xd = collapse_x(dx, phi, gx, gy, gz);
    Interp r;
    r.gap = collapse_yz(xa, by, bz) + phi0;
    r.g[0] = collapse_yz(xd, by, bz) * ih[0];
    r.g[1] = collapse_yz(xa, dy, bz) * ih[1];
    r.g[2] = collapse_yz(xa, by, dz) * ih[2];
    if (HESS)
    {
        float sx[4], sy[4], sz[4];
        hermite2(u, sx);
        hermite2(v, sy);
        hermite2(w, sz);
        const XColl xs = collapse_x(sx, phi, gx, gy, gz);
        r.H[0] = collapse_yz(xs, by, bz) * (ih[0] * ih[0]);
        r.H[1] = collapse_yz(xd, dy, bz) * (ih[0] * ih[1]);
        r.H[2] = collapse_yz(xd, by, dz) * (ih[0] * ih[2]);
        r.H[3] = collapse_yz(xa, sy, bz) * (ih[1] * ih[1]);
        r.H[4] = collapse_yz(xa, dy, dz) * (ih[1] * ih[2]);
        r.H[5] = collapse_yz(xa, by, sz) * (ih[2] * ih[2]);
    }
    else
    {
#pragma unroll
        for (int q = 0; q < 6; ++q) r.H[q] = 0.f;
    }
    return r;
}

__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }

// Trilinear (SdfOracle.cpp:551-583) over corner phi; optional mixed second
// derivatives (the diagonal ones are zero).
template <bool HESS>
__device__ __forceinline__ Interp trilinear(const float c[8], float u, float v, float w,
                                            const float ih[3])
{
    Interp r;
    const float c00 = lerpf(c[0], c[1], u), c10 = lerpf(c[2], c[3], u);
    const float c01 = lerpf(c[4], c[5], u), c11 = lerpf(c[6], c[7], u);
    r.gap = lerpf(lerpf(c00, c10, v), lerpf(c01, c11, v), w);
    // x differences at (j,k), y differences at (i,k), z differences at (i,j)
    const float dx00 = c[1] - c[0], dx10 = c[3] - c[2], dx01 = c[5] - c[4], dx11 = c[7] - c[6];
    const float dy00 = c[2] - c[0], dy10 = c[3] - c[1], dy01 = c[6] - c[4], dy11 = c[7] - c[5];
    const float dz00 = c[4] - c[0], dz10 = c[5] - c[1], dz01 = c[6] - c[2], dz11 = c[7] - c[3];
    r.g[0] = lerpf(lerpf(dx00, dx10, v), lerpf(dx01, dx11, v), w) * ih[0];
    r.g[1] = lerpf(lerpf(dy00, dy10, u), lerpf(dy01, dy11, u), w) * ih[1];
    r.g[2] = lerpf(lerpf(dz00, dz10, u), lerpf(dz01, dz11, u), v) * ih[2];
    r.H[0] = r.H[3] = r.H[5] = 0.f;
    if (HESS)
    {
        r.H[1] = lerpf(dx10 - dx00, dx11 - dx01, w) * (ih[0] * ih[1]);
        r.H[2] = lerpf(dx01 - dx00, dx11 - dx10, v) * (ih[0] * ih[2]);
        r.H[4] = lerpf(dy01 - dy00, dy11 - dy10, u) * (ih[1] * ih[2]);
    }
    else
    {
        r.H[1] = r.H[2] = r.H[4] = 0.f;
    }
    return r;
}

// ---------------------------------------------------------------------------
// one query of any mode (SdfOracle::queryFast and the per-mode queries,
// SdfOracle.cpp:226-432, 448-851, 932-1092)
// ---------------------------------------------------------------------------
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

// unit (the normalised gradient) is computed only when want_unit is set;
// otherwise it is left unset for Trilinear / Tricubic.
template <int MODE, bool SPARSE, int BD, bool HESS, int ST = 0>
__device__ __forceinline__ bool evaluate(const GridView& g, const double p[3], Interp& r,
                                         float unit[3], bool want_unit = true)
{
    const float h[3] = {(float)g.voxel[0], (float)g.voxel[1], (float)g.voxel[2]};
    const float ih[3] = {g.ih[0], g.ih[1], g.ih[2]};
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
            r = trilinear<HESS>(phi, c.u, c.v, c.w, ih);
            if (want_unit) unit_of(r.g, unit);
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
        else if (SPARSE && BD == 8 && g.phin_a32)
        {
            if (!gather_rows_b8<ST>(g, c, cs)) return false;
        }
        else
        {
            int64_t idx[8];
            if (!gather_corners<SPARSE, BD>(g, c, cs, idx)) return false;
        }
        if (MODE == SDFO_TRICUBIC)
        {
            r = tricubic<HESS>(cs, c.u, c.v, c.w, h, ih);
        }
        else
        {
            float phi[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) phi[q] = cs[q].x;
            r = trilinear<HESS>(phi, c.u, c.v, c.w, ih);
        }
        if (want_unit) unit_of(r.g, unit);
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

} // namespace sdfo
