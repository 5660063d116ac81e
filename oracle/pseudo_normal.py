"""NumPy restatement of the pseudo-normal sign rule (oracle).

TEST INFRASTRUCTURE ONLY.  The sign the builders use in
SDFO_SIGN_PSEUDONORMAL mode (no reference counterpart; the reference signs by
ray parity, KdTree.h:143-165): the angle-weighted pseudo-normals of Baerentzen
and Aanaes (IEEE TVCG 2005) -- vertex normals weighted by the corner angles,
edge normals summing the two face normals -- and, for each point, the normal
of the Voronoi region of its closest point on the nearest triangle.  The
closest point and its region follow closestPointOnTriangle
(KdTree.h:26-74) operation for operation in FP64, so squared distances equal
the builders' bit for bit; the nearest triangle is found by brute force
(lowest index on ties).
"""
from __future__ import annotations

import numpy as np

REGION_A, REGION_B, REGION_C, REGION_AB, REGION_AC, REGION_BC, REGION_FACE = range(7)


def pseudo_normals(verts, tris):
    """(T, 6, 3): unit normals of vertices a, b, c and edges ab, ac, bc of
    each triangle; degenerate triangles (|cross| <= 1e-15) add nothing."""
    v = np.asarray(verts, np.float64)
    t = np.asarray(tris, np.int64)
    P = v[t]  # (T,3,3)
    e1 = P[:, 1] - P[:, 0]
    e2 = P[:, 2] - P[:, 0]
    cr = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1], e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                   e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], 1)
    ln = np.sqrt(cr[:, 0] ** 2 + cr[:, 1] ** 2 + cr[:, 2] ** 2)
    ok = ln > 1e-15
    f = np.zeros_like(cr)
    f[ok] = cr[ok] / ln[ok, None]
    vn = np.zeros_like(v)
    for k in range(3):
        o, q1, q2 = P[:, k], P[:, (k + 1) % 3], P[:, (k + 2) % 3]
        u, w = q1 - o, q2 - o
        lu = np.sqrt(np.sum(u * u, 1))
        lw = np.sqrt(np.sum(w * w, 1))
        good = ok & (lu > 0) & (lw > 0)
        c = np.clip(np.sum(u * w, 1) / np.where(good, lu * lw, 1.0), -1.0, 1.0)
        ang = np.where(good, np.arccos(c), 0.0)
        np.add.at(vn, t[:, k], ang[:, None] * f)
    edges = [(0, 1), (0, 2), (1, 2)]
    keys = np.concatenate([np.sort(t[:, list(e)], 1) for e in edges])  # (3T, 2)
    uk, inv = np.unique(keys, axis=0, return_inverse=True)
    en = np.zeros((len(uk), 3))
    np.add.at(en, inv.reshape(-1), np.concatenate([f, f, f]))

    def unit(x):
        n = np.sqrt(np.sum(x * x, -1, keepdims=True))
        return np.where(n > 0, x / np.where(n > 0, n, 1.0), 0.0)

    out = np.zeros((len(t), 6, 3))
    for k in range(3):
        out[:, k] = unit(vn[t[:, k]])
    T = len(t)
    for k in range(3):
        out[:, 3 + k] = unit(en[inv.reshape(-1)[k * T:(k + 1) * T]])
    return out


def _dot(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def closest_points(p, a, b, c):
    """Ericson's closest point and its region for broadcast arrays (..., 3)."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = _dot(ab, ap), _dot(ac, ap)
    bp = p - b
    d3, d4 = _dot(ab, bp), _dot(ac, bp)
    vc = d1 * d4 - d3 * d2
    cp_ = p - c
    d5, d6 = _dot(ab, cp_), _dot(ac, cp_)
    vb = d5 * d2 - d1 * d6
    va = d3 * d6 - d5 * d4
    conds = [(d1 <= 0.0) & (d2 <= 0.0), (d3 >= 0.0) & (d4 <= d3), (vc <= 0.0) & (d1 >= 0.0) & (d3 <= 0.0),
             (d6 >= 0.0) & (d5 <= d6), (vb <= 0.0) & (d2 >= 0.0) & (d6 <= 0.0),
             (va <= 0.0) & ((d4 - d3) >= 0.0) & ((d5 - d6) >= 0.0)]
    region = np.select(conds, [REGION_A, REGION_B, REGION_AB, REGION_C, REGION_AC, REGION_BC], REGION_FACE)
    with np.errstate(divide="ignore", invalid="ignore"):
        v_ab = d1 / (d1 - d3)
        w_ac = d2 / (d2 - d6)
        w_bc = (d4 - d3) / ((d4 - d3) + (d5 - d6))
        denom = 1.0 / (va + vb + vc)
        v_f, w_f = vb * denom, vc * denom
    cp = a + ab * v_f[..., None] + ac * w_f[..., None]
    cp = np.where((region == REGION_A)[..., None], a, cp)
    cp = np.where((region == REGION_B)[..., None], b, cp)
    cp = np.where((region == REGION_C)[..., None], c, cp)
    cp = np.where((region == REGION_AB)[..., None], a + v_ab[..., None] * ab, cp)
    cp = np.where((region == REGION_AC)[..., None], a + w_ac[..., None] * ac, cp)
    cp = np.where((region == REGION_BC)[..., None], b + w_bc[..., None] * (c - b), cp)
    return cp, region


def signed_distance(verts, tris, pts, chunk=1024):
    """Pseudo-normal signed distance of each point: (sd, triangle, region)."""
    v = np.asarray(verts, np.float64)
    t = np.asarray(tris, np.int64)
    p = np.asarray(pts, np.float64).reshape(-1, 3)
    A, B, C = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    pn = pseudo_normals(v, t)
    e1, e2 = B - A, C - A
    cr = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1], e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                   e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], 1)
    ln = np.sqrt(_dot(cr, cr))
    fn = np.where((ln > 1e-15)[:, None], cr / np.where(ln > 1e-15, ln, 1.0)[:, None], [0.0, 0.0, 1.0])
    sd = np.zeros(len(p))
    tri = np.zeros(len(p), np.int64)
    reg = np.zeros(len(p), np.int64)
    for s in range(0, len(p), chunk):
        q = p[s:s + chunk, None, :]
        cp, region = closest_points(q, A[None], B[None], C[None])
        d = q - cp
        sq = _dot(d, d)
        k = np.argmin(sq, 1)
        rows = np.arange(len(k))
        cpk = cp[rows, k]
        rk = region[rows, k]
        n = np.where((rk < REGION_FACE)[:, None], pn[k, np.minimum(rk, 5)], fn[k])
        dist = np.sqrt(sq[rows, k])
        side = _dot(p[s:s + chunk] - cpk, n) >= 0.0
        sd[s:s + chunk] = np.where(side, dist, -dist)
        tri[s:s + chunk] = k
        reg[s:s + chunk] = rk
    return sd, tri, reg
