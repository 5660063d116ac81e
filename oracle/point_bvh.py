"""NumPy restatement of the prototype's point broad phase (oracle).

TEST INFRASTRUCTURE ONLY.  Follows prototype/src/geometry/bvh.py and the
culling steps of prototype/src/dynamics/contacts_sdf.py:
  - AABB_BVH._build (bvh.py:27-60): node box = min/max of its points; leaf
    when n <= leaf_size; else the longest axis (first on ties), split at the
    box midpoint, points <= mid left in their order; if a side is empty, a
    median split of the points sorted along the axis (stable sort here)
  - AABB_BVH.query (bvh.py:62-80): all points when the query box encloses
    the root box; else the points of the leaves a stack traversal reaches
    (right child popped first), skipping nodes with max < qmin or min > qmax
    on any axis
  - evaluate's cull (contacts_sdf.py:244-298): query box
    RA^T (bmin - rA) -+ max(narrow_margin, 0.05), every point when nothing is
    kept, then the narrow filter |Y_z| < narrow_margin
  - measure_pair (contacts_sdf.py:171-214) over the BVH-kept points.
Pinned against the prototype itself by tests/golden (make_golden.py runs
AABB_BVH, SDFContactEngine.evaluate and measure_pair).
"""
from __future__ import annotations

import numpy as np

from oracle.contact_port import evaluate_pose


def build(X, leaf_size=16):
    """Leaves in the query's visiting order: (order, starts, boxes (L,6))."""
    X = np.asarray(X, np.float64)
    leaves = []

    def node(idx):
        pts = X[idx]
        lo, hi = pts.min(0), pts.max(0)
        if len(idx) <= leaf_size:
            leaves.append((idx, np.concatenate([lo, hi])))
            return
        axis = int(np.argmax(hi - lo))
        mid = (lo[axis] + hi[axis]) * 0.5
        left, right = idx[pts[:, axis] <= mid], idx[pts[:, axis] > mid]
        if len(left) == 0 or len(right) == 0:
            s = np.argsort(pts[:, axis], kind="stable")
            half = len(idx) // 2
            left, right = idx[s[:half]], idx[s[half:]]
        node(right)  # popped first by the query's stack
        node(left)

    if len(X):
        node(np.arange(len(X)))
    order = np.concatenate([l[0] for l in leaves]).astype(np.int32) if leaves else np.zeros(0, np.int32)
    starts = np.concatenate([[0], np.cumsum([len(l[0]) for l in leaves])]).astype(np.int32)
    boxes = np.array([l[1] for l in leaves]).reshape(-1, 6)
    return order, starts, boxes


def query(X, order, starts, boxes, qmin, qmax):
    """AABB_BVH.query(qmin, qmax) on the leaves (a leaf is reached iff it
    overlaps: every ancestor's box contains it)."""
    X = np.asarray(X, np.float64)
    lo, hi = X.min(0), X.max(0)
    if np.all(qmin <= lo) and np.all(qmax >= hi):
        return np.arange(len(X), dtype=np.int32)
    keep = ~(np.any(boxes[:, 3:] < qmin, axis=1) | np.any(boxes[:, :3] > qmax, axis=1))
    parts = [order[starts[l]:starts[l + 1]] for l in np.nonzero(keep)[0]]
    return np.concatenate(parts).astype(np.int32) if parts else np.zeros(0, np.int32)


def cull_indices(X, bvh, bmin, bmax, rA, RA, narrow_margin):
    margin = max(narrow_margin, 0.05)
    qmin = RA.T @ (bmin - rA) - margin
    qmax = RA.T @ (bmax - rA) + margin
    idx = query(X, *bvh, qmin, qmax)
    if len(idx) == 0:
        idx = np.arange(len(X), dtype=np.int32)
    return idx


def evaluate_culled(query_batch, Xq, wq, bvh, bmin, bmax, narrow_margin, rA, RA, vA, wA, rB, RB,
                    vB, wB, k, order, damping, mu, regularizer):
    """F_A, tau_A of SDFContactEngine.evaluate with its culling."""
    idx = cull_indices(Xq, bvh, bmin, bmax, rA, RA, narrow_margin)
    Y = ((RB.T @ RA) @ Xq[idx].T + (RB.T @ (rA - rB))[:, None]).T
    keep = idx[np.abs(Y[:, 2]) < narrow_margin]
    if len(keep) == 0:
        return np.zeros(3), np.zeros(3)
    F, tau, _, _ = evaluate_pose(query_batch, Xq[keep], wq[keep], rA, RA, vA, wA, rB, RB, vB, wB,
                                 k, order, damping, mu, regularizer)
    return F, tau


def measure(query_batch, Xq, bvh, bmin, bmax, narrow_margin, rA, RA, vA, wA, rB, RB, vB, wB,
            tie_tol=0.0):
    """measure_pair: (gap, penetration, normal_velocity, min_point_index,
    active_count, valid_count), plus a function giving the normal velocity at
    any position of the kept list and the positions whose gap is within
    tie_tol of the minimum (exactly equal gaps in exact arithmetic, e.g. a
    flat face over a plane, are ordered by rounding)."""
    idx = cull_indices(Xq, bvh, bmin, bmax, rA, RA, narrow_margin)
    Y = ((RB.T @ RA) @ Xq[idx].T + (RB.T @ (rA - rB))[:, None]).T
    g, raw, gn, unit, valid = query_batch(Y)

    def vn_at(mi):
        xw = rA + RA @ Xq[idx[mi]]
        n = RB @ unit[mi]
        nn = np.linalg.norm(n)
        if nn > 1e-30:
            n = n / nn
        uA = vA + np.cross(wA, xw - rA)
        uB = vB + np.cross(wB, xw - rB)
        return float(np.dot(uA - uB, n))

    if not np.any(valid):
        return (np.inf, 0.0, 0.0, -1, 0, 0), vn_at, np.zeros(0, np.int64)
    vi = np.nonzero(valid)[0]
    mi = int(vi[int(np.argmin(g[valid]))])
    gmin = float(g[mi])
    ties = vi[g[vi] <= gmin + tie_tol]
    return ((gmin, max(0.0, -gmin), vn_at(mi), mi, int(np.sum(valid & (g < 0.0))),
             int(np.sum(valid))), vn_at, ties)
