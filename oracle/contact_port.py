"""NumPy restatement of SDFContactEngine.evaluate's force law (oracle).

TEST INFRASTRUCTURE ONLY.  Follows prototype/src/dynamics/contacts_sdf.py:
  - marker-free transform Y = R_B^T R_A X + R_B^T (r_A - r_B)   (:275-286)
  - valid_mask = valid & (k max(-g,0)^n > 1e-30)               (:329)
  - rg = R_B grad g, fn = p rg, p_hat = p |grad g|             (:338-351)
  - damping c (-(u_A - u_B).rg) rg where g < 0                 (:353-361)
  - friction -mu p_hat u_t / sqrt(|u_t|^2 + reg^2)             (:363-377)
  - F_A = sum w f, tau_A = sum w (x - r_A) x f                 (:379-381)
The culling steps of evaluate (AABB broad phase, point BVH, |Y_z| < margin
narrow filter) only drop points that produce no force when their margins
cover the grid, so they are not restated.  Pinned against the prototype
itself by tests/golden (make_golden.py runs SDFContactEngine.evaluate).
"""
from __future__ import annotations

import numpy as np


def evaluate_pose(query_batch, Xq, wq, rA, RA, vA, wA, rB, RB, vB, wB, k, order, damping, mu,
                  regularizer, freeze=None):
    """One pose.  query_batch(Y) -> (g, raw_grad, grad_norm, unit, valid) in
    body-B coordinates (FP64).  ``freeze`` = (mask, g0, grad0) replaces the
    query with a first-order model around a reference pose (used to take
    finite differences of the smooth branch only); returns F_A, tau_A and the
    per-point (g, valid_mask) actually used."""
    R_sdf = RB.T @ RA
    t_sdf = RB.T @ (rA - rB)
    Y = (R_sdf @ Xq.T + t_sdf[:, None]).T
    g, raw_grad, grad_norm, unit, valid = query_batch(Y)
    p_all = k * np.maximum(-g, 0.0) ** order
    valid_mask = valid & (p_all > 1e-30)
    if freeze is not None:
        valid_mask = freeze
    if not np.any(valid_mask):
        return np.zeros(3), np.zeros(3), g, valid_mask
    gv = g[valid_mask]
    rg_local = raw_grad[valid_mask]
    gn = grad_norm[valid_mask]
    p = k * np.maximum(-gv, 0.0) ** order
    rg = (RB @ rg_local.T).T
    xw = (rA[:, None] + RA @ Xq[valid_mask].T).T
    wv = wq[valid_mask]
    off_A = xw - rA[None, :]
    fn = p[:, None] * rg
    p_hat = p * gn
    uA = vA[None, :] + np.cross(wA[None, :], off_A)
    uB = vB[None, :] + np.cross(wB[None, :], xw - rB[None, :])
    u_rel = uA - uB
    if damping > 0:
        vn = np.sum(u_rel * rg, axis=1)
        # the damping switch g < 0 is a step; with the active set frozen it is
        # kept on for every frozen point (all had g < 0 at the base pose)
        damp_on = np.ones_like(gv, bool) if freeze is not None else (gv < 0.0)
        fn = fn + damping * (-vn)[:, None] * rg * damp_on[:, None]
    un = rg / np.maximum(gn[:, None], 1e-30)
    udotn = np.sum(u_rel * un, axis=1, keepdims=True)
    u_t = u_rel - udotn * un
    denom = np.sqrt(np.linalg.norm(u_t, axis=1) ** 2 + regularizer ** 2)
    ft = np.zeros_like(fn)
    act = mu * p_hat > 0
    if np.any(act):
        ft[act] = -mu * p_hat[act, None] * u_t[act] / denom[act, None]
    fq = fn + ft
    F = np.sum(wv[:, None] * fq, axis=0)
    tau = np.sum(wv[:, None] * np.cross(off_A, fq), axis=0)
    return F, tau, g, valid_mask


def rotvec(theta):
    a = np.linalg.norm(theta)
    if a == 0.0:
        return np.eye(3)
    k = theta / a
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K


def fd_jacobian_pose(query_batch, Xq, wq, rA, RA, vA, wA, rB, RB, vB, wB, prm, h_lin=1e-7,
                     h_ang=1e-6, freeze_active=True):
    """Central-difference 6x6 d(F,tau)/d(dx,dtheta).  With freeze_active the
    active point set of the base pose is kept for the perturbed poses (the
    derivative of the smooth branch, which is what forward-mode AD gives)."""
    F0, t0, g0, mask0 = evaluate_pose(query_batch, Xq, wq, rA, RA, vA, wA, rB, RB, vB, wB, **prm)
    J = np.zeros((6, 6))
    for j in range(6):
        cols = []
        for s in (1.0, -1.0):
            r2, R2 = rA.copy(), RA.copy()
            if j < 3:
                r2[j] += s * h_lin
            else:
                th = np.zeros(3)
                th[j - 3] = s * h_ang
                R2 = rotvec(th) @ RA
            F, tau, _, _ = evaluate_pose(query_batch, Xq, wq, r2, R2, vA, wA, rB, RB, vB, wB,
                                         freeze=mask0 if freeze_active else None, **prm)
            cols.append(np.concatenate([F, tau]))
        h = h_lin if j < 3 else h_ang
        J[:, j] = (cols[0] - cols[1]) / (2.0 * h)
    return np.concatenate([F0, t0]), J
