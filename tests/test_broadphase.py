"""The quadrature broad phase: the point hierarchy (AABB_BVH,
prototype/src/geometry/bvh.py) and SDFContactEngine's culling in evaluate /
measure_pair (prototype/src/dynamics/contacts_sdf.py:171-298), against
fixtures the prototype itself produced (tests/golden/make_golden.py)."""
import ctypes

import numpy as np
import pytest

from conftest import golden

CLOUDS = ["torus", "random", "small"]


def _pair_bvh(X):
    """Hierarchy built by the library (sdfo_contact_pair_create, no grid)."""
    from sdfo import _native as N

    lib = N.load()
    X = np.ascontiguousarray(X, np.float64)
    w = np.ones(len(X))
    out = ctypes.c_void_p()
    N.check(lib.sdfo_contact_pair_create(None, X.ctypes.data_as(ctypes.c_void_p),
                                         w.ctypes.data_as(ctypes.c_void_p), len(X), 1, 0.01, 16,
                                         ctypes.byref(out)))
    try:
        nl = ctypes.c_int32()
        N.check(lib.sdfo_contact_pair_export_bvh(out, ctypes.byref(nl), None, None, None))
        o = np.zeros(len(X), np.int32)
        s = np.zeros(nl.value + 1, np.int32)
        b = np.zeros((nl.value, 6))
        N.check(lib.sdfo_contact_pair_export_bvh(out, None, o.ctypes.data_as(ctypes.c_void_p),
                                                 s.ctypes.data_as(ctypes.c_void_p),
                                                 b.ctypes.data_as(ctypes.c_void_p)))
    finally:
        lib.sdfo_contact_pair_destroy(out)
    return o, s, b


@pytest.mark.parametrize("cloud", CLOUDS)
def test_point_bvh_oracle_matches_prototype(cloud):
    from oracle import point_bvh as B

    d = golden("point_bvh.npz")
    X = d[f"{cloud}_points"]
    o, s, b = B.build(X)
    np.testing.assert_array_equal(o, d[f"{cloud}_order"])
    np.testing.assert_array_equal(s, d[f"{cloud}_starts"])
    np.testing.assert_array_equal(b, d[f"{cloud}_boxes"])
    rs, res = d[f"{cloud}_result_starts"], d[f"{cloud}_results"]
    for k in range(len(d[f"{cloud}_qmin"])):
        r = B.query(X, o, s, b, d[f"{cloud}_qmin"][k], d[f"{cloud}_qmax"][k])
        np.testing.assert_array_equal(r, res[rs[k]:rs[k + 1]])


@pytest.mark.parametrize("cloud", CLOUDS)
def test_library_point_bvh_matches_prototype(cloud):
    d = golden("point_bvh.npz")
    o, s, b = _pair_bvh(d[f"{cloud}_points"])
    np.testing.assert_array_equal(o, d[f"{cloud}_order"])
    np.testing.assert_array_equal(s, d[f"{cloud}_starts"])
    np.testing.assert_array_equal(b, d[f"{cloud}_boxes"])


def _slab():
    g = golden("engine_culling.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    return g, spec


def _qb(spec, phi, normal):
    from oracle import interp_np

    def qb(Y):
        gap, grad, valid, _ = interp_np.query(spec, phi, normal, 2, Y)
        gn = np.linalg.norm(grad, axis=1)
        unit = np.zeros_like(grad)
        unit[:, 2] = 1.0
        ok = valid & (gn > 1e-30)
        unit[ok] = grad[ok] / gn[ok, None]
        return gap, grad, gn, unit, valid

    return qb


def _split(pose):
    return pose[:3], pose[3:12].reshape(3, 3), pose[12:15], pose[15:18]


def test_culling_oracle_matches_prototype():
    """oracle/point_bvh evaluate_culled / measure vs the prototype engine with
    its default culling (register_pair narrow_margin 0.01)."""
    from oracle import point_bvh as B

    g, spec = _slab()
    qb = _qb(spec, g["phi"], g["normal"])
    X = g["quad_x"]
    w = g["quad_w"] / g["quad_w"].sum()
    bvh = B.build(X)
    nm = float(g["narrow_margin"])
    prm = dict(k=float(g["k"]), order=float(g["order"]), damping=float(g["damping"]),
               mu=float(g["mu"]), regularizer=float(g["reg"]))
    in_contact = 0
    for pose, pb, ref_f, ref_m in zip(g["poses"], g["body_b"], g["forces"], g["measure"]):
        rA, RA, vA, wA = _split(pose)
        rB, RB, vB, wB = _split(pb)
        F, tau = B.evaluate_culled(qb, X, w, bvh, g["bmin"], g["bmax"], nm, rA, RA, vA, wA, rB, RB,
                                   vB, wB, **prm)
        scale = max(np.abs(ref_f[:6]).max(), 1e-12)
        assert np.abs(np.concatenate([F, tau]) - ref_f[:6]).max() <= 1e-9 * scale
        m, vn_at, ties = B.measure(qb, X, bvh, g["bmin"], g["bmax"], nm, rA, RA, vA, wA, rB, RB,
                                   vB, wB, tie_tol=1e-12)
        if np.isinf(ref_m[0]):
            assert np.isinf(m[0]) and m[3:] == (-1, 0, 0)
        else:
            assert abs(m[0] - ref_m[0]) <= 1e-12 and abs(m[1] - ref_m[1]) <= 1e-12
            assert m[4:] == tuple(int(x) for x in ref_m[4:])
            # the argmin is the reference's, or one of a set of gaps equal up
            # to rounding (a flat face over the plane)
            assert int(ref_m[3]) in ties
            assert abs(vn_at(int(ref_m[3])) - ref_m[2]) <= 1e-9 * max(1.0, abs(ref_m[2]))
        in_contact += np.abs(ref_f[:3]).max() > 0
    assert in_contact >= 10


# --------------------------------------------------------------------- GPU
def _gpu_batch(g, spec, narrow_margin=0.01, mode=2):
    from sdfo import SdfGrid
    from sdfo.contact import ContactBatch

    grid = SdfGrid.from_dense(spec, g["phi"], g["normal"])
    cb = ContactBatch(grid, g["quad_x"], g["quad_w"], stiffness=float(g["k"]),
                      order=float(g["order"]), damping=float(g["damping"]), friction=float(g["mu"]),
                      regularizer=float(g["reg"]), mode=mode, narrow_margin=narrow_margin)
    return grid, cb


def _states(poses):
    from sdfo.contact import pack_states

    return pack_states(poses[:, :3], poses[:, 3:12].reshape(-1, 3, 3), poses[:, 12:15], poses[:, 15:18])


@pytest.mark.gpu
def test_culled_contact_matches_prototype(cuda):
    """ContactBatch(narrow_margin=0.01).evaluate / measure on the GPU vs the
    prototype engine: forces within 1e-5 of the pose's force scale (FP32
    grid and points); measures: counts exact, gap within 1e-6 (FP32
    interpolation), the argmin the reference's point or one tied with it up
    to FP32 rounding, the normal velocity at that point within 1e-5."""
    from oracle import point_bvh as B

    g, spec = _slab()
    grid, cb = _gpu_batch(g, spec)
    qb = _qb(spec, g["phi"].astype(np.float32).astype(np.float64),
             g["normal"].astype(np.float32).astype(np.float64))
    bvh = B.build(g["quad_x"])
    for k in range(len(g["poses"])):
        pa = _states(g["poses"][k:k + 1])
        pb = _states(g["body_b"][k:k + 1])[0]
        ft = cb.evaluate(pa, pb).cpu().numpy()[0]
        m = {key: v.cpu().numpy()[0] for key, v in cb.measure(pa, pb).items()}
        ref_f, ref_m = g["forces"][k], g["measure"][k]
        scale = max(np.abs(ref_f[:6]).max(), 1e-9)
        assert np.abs(ft - ref_f[:6]).max() <= 1e-5 * scale, (k, ft, ref_f[:6])
        assert int(m["valid_count"]) == int(ref_m[5]) and int(m["active_count"]) == int(ref_m[4]), k
        if np.isinf(ref_m[0]):
            assert np.isinf(m["gap"]) and int(m["min_point_index"]) == -1
            continue
        assert abs(m["gap"] - ref_m[0]) <= 1e-6, k
        # the argmin: the reference's point, or one whose gap equals the
        # minimum up to FP32 rounding (then its own normal velocity)
        rA, RA, vA, wA = _split(g["poses"][k])
        rB, RB, vB, wB = _split(g["body_b"][k])
        _, vn_at, ties = B.measure(qb, g["quad_x"].astype(np.float32).astype(np.float64), bvh,
                                   g["bmin"], g["bmax"], 0.01, rA, RA, vA, wA, rB, RB, vB, wB,
                                   tie_tol=2e-6)
        mi = int(m["min_point_index"])
        assert mi == int(ref_m[3]) or mi in ties, k
        assert abs(m["normal_velocity"] - vn_at(mi)) <= 1e-5 * max(1.0, abs(vn_at(mi))), k


@pytest.mark.gpu
def test_culled_contact_batch_vs_oracle(cuda):
    """256 random poses (any rotation, near the plane, some far or over the
    grid's edge, body B moved) in one launch vs the oracle on the same
    FP32-rounded grid."""
    from oracle import point_bvh as B

    from sdfo.contact import pack_states

    g, spec = _slab()
    grid, cb = _gpu_batch(g, spec)
    phi32 = g["phi"].astype(np.float32).astype(np.float64)
    n32 = g["normal"].astype(np.float32).astype(np.float64)
    qb = _qb(spec, phi32, n32)
    X = g["quad_x"].astype(np.float32).astype(np.float64)
    w = (g["quad_w"] / g["quad_w"].sum()).astype(np.float32).astype(np.float64)
    bvh = B.build(g["quad_x"])
    rng = np.random.default_rng(41)
    P = 256
    r = np.zeros((P, 3))
    R = np.zeros((P, 3, 3))
    for p in range(P):
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        ang = rng.uniform(0, np.pi) if p % 2 else rng.uniform(0, 0.1)
        K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
        R[p] = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
        z = -(R[p] @ g["quad_x"].T)[2].min() - rng.uniform(0.0, 0.002)
        r[p] = [rng.uniform(-0.2, 0.2), rng.uniform(-0.2, 0.2), z if p % 7 else 0.05]
    v = rng.normal(size=(P, 3)) * 0.05
    om = rng.normal(size=(P, 3)) * 0.5
    rB, RB = np.array([0.004, -0.003, 0.001]), np.eye(3)
    pa = pack_states(r, R, v, om)
    pb = pack_states(rB[None], RB[None])[0]
    ft = cb.evaluate(pa, pb).cpu().numpy()
    ms = {k: x.cpu().numpy() for k, x in cb.measure(pa, pb).items()}
    prm = dict(k=float(g["k"]), order=float(g["order"]), damping=float(g["damping"]),
               mu=float(g["mu"]), regularizer=float(g["reg"]))
    refs = []
    for p in range(P):
        F, tau = B.evaluate_culled(qb, X, w, bvh, g["bmin"], g["bmax"], 0.01, r[p], R[p], v[p], om[p],
                                   rB, RB, np.zeros(3), np.zeros(3), **prm)
        refs.append(np.concatenate([F, tau]))
    # a barely touching pose's force is set by FP32 gap rounding: its floor is
    # 1e-3 of the batch's largest force
    floor = 1e-3 * np.abs(np.array(refs)).max()
    hits = 0
    for p in range(P):
        ref = refs[p]
        scale = max(np.abs(ref).max(), floor)
        assert np.abs(ft[p] - ref).max() <= 1e-5 * scale, (p, ft[p], ref)
        m, _, _ = B.measure(qb, X, bvh, g["bmin"], g["bmax"], 0.01, r[p], R[p], v[p], om[p], rB,
                            RB, np.zeros(3), np.zeros(3))
        assert (int(ms["valid_count"][p]), int(ms["active_count"][p])) == (m[5], m[4]), p
        if m[5]:
            assert abs(ms["gap"][p] - m[0]) <= 1e-6, p
        hits += np.abs(ref).max() > 0
    assert hits >= 50


@pytest.mark.gpu
def test_culling_with_wide_margin_equals_plain_evaluation(cuda):
    """A narrow margin that keeps every point gives the plain kernel's forces
    and Jacobian (summed in another point order: within 1e-12)."""
    g, spec = _slab()
    grid, plain = _gpu_batch(g, spec, narrow_margin=None)
    _, wide = _gpu_batch(g, spec, narrow_margin=1e9)
    pa = _states(g["poses"])
    pb = _states(g["body_b"][:1])[0]
    f0, j0 = plain.evaluate(pa, pb, jacobian=True)
    f1, j1 = wide.evaluate(pa, pb, jacobian=True)
    sf = max(float(f0.abs().max()), 1e-9)
    sj = max(float(j0.abs().max()), 1e-9)
    assert float((f0 - f1).abs().max()) <= 1e-12 * sf
    assert float((j0 - j1).abs().max()) <= 1e-12 * sj
