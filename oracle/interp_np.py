"""Vectorised FP64 NumPy restatement of the Trilinear and Tricubic queries on a
dense grid, with an optional fixed cell per point (oracle).

TEST INFRASTRUCTURE ONLY.  Same interpolants as SdfOracle::trilinearQuery
(SdfOracle.cpp:524-596) and tricubicQuery (SdfOracle.cpp:932-1092); it is
pinned against the C restatement (oracle/sdfo_port.cpp) by a CPU test.  The
``cells`` argument evaluates each point with the polynomial of a given cell
(extrapolating slightly outside it), so finite differences taken with the
cells frozen differentiate one smooth piece -- the quantity forward-mode AD
computes.
"""
from __future__ import annotations

import numpy as np


def _h(t):
    return np.stack([t * t * (2 * t - 3) + 1, t * (t * (t - 2) + 1), t * t * (3 - 2 * t),
                     t * t * (t - 1)], -1)


def _dh(t):
    return np.stack([6 * t * (t - 1), t * (3 * t - 4) + 1, 6 * t * (1 - t), t * (3 * t - 2)], -1)


def query(spec, phi, normal, mode, Y, cells=None):
    """spec: dict(bmin, voxel, shape); phi (N,), normal (N,3) FP64 x-fastest.
    mode 2 = Trilinear, 3 = Tricubic.  Returns gap, grad (raw), valid, cells."""
    Y = np.asarray(Y, np.float64).reshape(-1, 3)
    bmin = np.asarray(spec["bmin"], np.float64)
    vox = np.asarray(spec["voxel"], np.float64)
    nx, ny, nz = [int(s) for s in spec["shape"]]
    f = (Y - bmin) / vox - 0.5
    if cells is None:
        with np.errstate(invalid="ignore"):
            ok = np.all(np.isfinite(f), axis=1)
            fl = np.floor(np.where(np.isfinite(f), f, 0.0)).astype(np.int64)
        valid = ok & (fl[:, 0] >= 0) & (fl[:, 0] + 1 < nx) & (fl[:, 1] >= 0) & (fl[:, 1] + 1 < ny) \
            & (fl[:, 2] >= 0) & (fl[:, 2] + 1 < nz)
        cells = fl
    else:
        cells = np.asarray(cells, np.int64)
        valid = np.all(np.isfinite(f), axis=1) & (cells[:, 0] >= 0) & (cells[:, 0] + 1 < nx) & \
            (cells[:, 1] >= 0) & (cells[:, 1] + 1 < ny) & (cells[:, 2] >= 0) & (cells[:, 2] + 1 < nz)
    u = f - cells
    c = np.where(valid[:, None], cells, 0)
    idx = np.empty((len(Y), 8), np.int64)
    for q in range(8):
        i = c[:, 0] + (q & 1)
        j = c[:, 1] + ((q >> 1) & 1)
        k = c[:, 2] + (q >> 2)
        idx[:, q] = i + nx * (j + ny * k)
    P = phi[idx]
    gap = np.zeros(len(Y))
    grad = np.zeros((len(Y), 3))
    if mode == 2:
        w = np.empty((len(Y), 8))
        dw = np.empty((len(Y), 8, 3))
        for q in range(8):
            bi, bj, bk = q & 1, (q >> 1) & 1, q >> 2
            wx = u[:, 0] if bi else 1 - u[:, 0]
            wy = u[:, 1] if bj else 1 - u[:, 1]
            wz = u[:, 2] if bk else 1 - u[:, 2]
            sx, sy, sz = (1.0 if bi else -1.0), (1.0 if bj else -1.0), (1.0 if bk else -1.0)
            w[:, q] = wx * wy * wz
            dw[:, q, 0] = sx * wy * wz / vox[0]
            dw[:, q, 1] = wx * sy * wz / vox[1]
            dw[:, q, 2] = wx * wy * sz / vox[2]
        gap = np.sum(w * P, 1)
        grad = np.einsum("nqa,nq->na", dw, P)
    else:
        N = normal[idx]  # (n, 8, 3)
        G = N * vox[None, None, :]
        H = [_h(u[:, a]) for a in range(3)]
        D = [_dh(u[:, a]) for a in range(3)]
        for q in range(8):
            b = [q & 1, (q >> 1) & 1, q >> 2]
            v0 = [H[a][:, 2 * b[a]] for a in range(3)]
            v1 = [H[a][:, 2 * b[a] + 1] for a in range(3)]
            d0 = [D[a][:, 2 * b[a]] for a in range(3)]
            d1 = [D[a][:, 2 * b[a] + 1] for a in range(3)]
            gap += v0[0] * v0[1] * v0[2] * P[:, q] + v1[0] * v0[1] * v0[2] * G[:, q, 0] \
                + v0[0] * v1[1] * v0[2] * G[:, q, 1] + v0[0] * v0[1] * v1[2] * G[:, q, 2]
            for a in range(3):
                e0 = [d0[x] if x == a else v0[x] for x in range(3)]
                e1x = d1[0] if a == 0 else v1[0]
                e1y = d1[1] if a == 1 else v1[1]
                e1z = d1[2] if a == 2 else v1[2]
                grad[:, a] += (e0[0] * e0[1] * e0[2] * P[:, q] + e1x * e0[1] * e0[2] * G[:, q, 0]
                               + e0[0] * e1y * e0[2] * G[:, q, 1]
                               + e0[0] * e0[1] * e1z * G[:, q, 2]) / vox[a]
    gap = np.where(valid, gap, 0.0)
    grad = np.where(valid[:, None], grad, 0.0)
    return gap, grad, valid, cells


def trilinear_hessian(spec, phi, Y):
    """Hessian (N,3,3) of the trilinear interpolant of query() mode 2 at Y
    (its cell's bilinear mixed partials; the diagonal is zero); zero where
    the point is invalid.  Used by the exact Newton tangent of the BE
    restatement."""
    Y = np.asarray(Y, np.float64).reshape(-1, 3)
    bmin = np.asarray(spec["bmin"], np.float64)
    vox = np.asarray(spec["voxel"], np.float64)
    nx, ny, nz = [int(s) for s in spec["shape"]]
    f = (Y - bmin) / vox - 0.5
    with np.errstate(invalid="ignore"):
        ok = np.all(np.isfinite(f), axis=1)
        c = np.floor(np.where(np.isfinite(f), f, 0.0)).astype(np.int64)
    valid = ok & (c[:, 0] >= 0) & (c[:, 0] + 1 < nx) & (c[:, 1] >= 0) & (c[:, 1] + 1 < ny) \
        & (c[:, 2] >= 0) & (c[:, 2] + 1 < nz)
    u = f - c
    c = np.where(valid[:, None], c, 0)

    def P(di, dj, dk):
        return phi[(c[:, 0] + di) + nx * ((c[:, 1] + dj) + ny * (c[:, 2] + dk))]

    p000, p100, p010, p110 = P(0, 0, 0), P(1, 0, 0), P(0, 1, 0), P(1, 1, 0)
    p001, p101, p011, p111 = P(0, 0, 1), P(1, 0, 1), P(0, 1, 1), P(1, 1, 1)
    hxy = ((p110 - p010 - p100 + p000) * (1 - u[:, 2]) + (p111 - p011 - p101 + p001) * u[:, 2]) \
        / (vox[0] * vox[1])
    hxz = ((p101 - p001 - p100 + p000) * (1 - u[:, 1]) + (p111 - p011 - p110 + p010) * u[:, 1]) \
        / (vox[0] * vox[2])
    hyz = ((p011 - p001 - p010 + p000) * (1 - u[:, 0]) + (p111 - p101 - p110 + p100) * u[:, 0]) \
        / (vox[1] * vox[2])
    H = np.zeros((len(Y), 3, 3))
    H[:, 0, 1] = H[:, 1, 0] = hxy
    H[:, 0, 2] = H[:, 2, 0] = hxz
    H[:, 1, 2] = H[:, 2, 1] = hyz
    H[~valid] = 0.0
    return H
