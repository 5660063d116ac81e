"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a container where the reference checkout is present:

    make -C oracle ref port
    python tests/golden/make_golden.py [--reference PATH]

PATH defaults to $SDFO_REFERENCE_ROOT, else a directory named ``reference``
beside this repository.

Sources of truth (nothing here is restated):
  * the reference C++ SdfOracle sources, compiled unmodified into
    oracle/_ref/libsdfo_ref.so (oracle/Makefile; Eigen3 is absent, so they
    compile against the Eigen-API subset in oracle/eigen_shim): SdfBuilder::
    build / buildSparse, SdfOracle::queryFast, KdTree::findSignedNearest,
    saveSdf / saveSparseSdf;
  * the reference Python prototype imported from the checkout:
    TrilinearSDFGrid.query_batch (prototype/src/sdf_grid.py) and
    SDFContactEngine.evaluate (prototype/src/dynamics/contacts_sdf.py).
Inputs are the procedural meshes of sdfo.meshes with fixed seeds.
"""
from __future__ import annotations

import argparse
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "sdf-contact-module_b200"))

from oracle import ref  # noqa: E402
from sdfo import meshes as M  # noqa: E402

SETUP_CASES = [
    # (mesh name, build kwargs)
    ("cube", dict(padding=0.1, voxel_size=0.0, target_resolution=64, max_resolution=64)),
    ("cube", dict(padding=4 * (0.1 / 56) / (0.1 * 3 ** 0.5), voxel_size=0.1 / 56,
                  target_resolution=64, max_resolution=64)),
    ("cyl", dict(padding=0.1, voxel_size=0.0, target_resolution=128, max_resolution=128)),
    ("cyl", dict(padding=0.1, voxel_size=0.0, target_resolution=96, max_resolution=96)),
    ("cyl", dict(padding=0.25, voxel_size=0.0, target_resolution=200, max_resolution=512)),
    ("gear", dict(padding=0.1, voxel_size=0.0, target_resolution=192, max_resolution=192)),
    ("torus", dict(padding=0.0, voxel_size=0.0, target_resolution=40, max_resolution=2048)),
]


def meshes():
    return {
        "cube": M.cube(0.1),
        "cyl": M.hollow_cylinder(0.05, 0.04, 0.02, n_az=64, n_vert=4),
        "torus": M.torus(0.05, 0.01, 48, 12),
        "gear": M.gear_prism(24, 0.05, 0.01, 3000),
    }


def query_points(info, n, seed):
    rng = np.random.default_rng(seed)
    lo = info["bmin"] - 0.05 * (info["bmax"] - info["bmin"])
    hi = info["bmax"] + 0.05 * (info["bmax"] - info["bmin"])
    pts = rng.uniform(lo, hi, (n, 3))
    # exact voxel centres and cell corners exercise the rounding / floor rules
    ijk = rng.integers(0, np.array(info["shape"]), (n // 8, 3))
    pts[: n // 8] = info["bmin"] + info["voxel"] * (ijk + 0.5)
    pts[n // 8: n // 4] = info["bmin"] + info["voxel"] * ijk
    return pts.astype(np.float32).astype(np.float64)


def ref_queries(g, pts):
    out = {}
    for mode in range(4):
        gap, nrm, wit, val = g.query(mode, pts)
        out[f"q{mode}_gap"] = gap
        out[f"q{mode}_normal"] = nrm
        out[f"q{mode}_witness"] = wit
        out[f"q{mode}_valid"] = val
    return out


def main():
    ap = argparse.ArgumentParser()
    default_ref = os.environ.get("SDFO_REFERENCE_ROOT") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference")
    ap.add_argument("--reference", default=default_ref)
    ap.add_argument("--only", choices=["all", "contact_aware", "broadphase", "be"], default="all")
    a = ap.parse_args()
    ms = meshes()
    if a.only == "contact_aware":
        _contact_aware_fixtures(ms)
        print("contact-aware fixtures written to", HERE)
        return
    if a.only == "broadphase":
        _broadphase_fixtures(a.reference)
        print("broad-phase fixtures written to", HERE)
        return
    if a.only == "be":
        _be_fixtures(a.reference)
        print("BE fixtures written to", HERE)
        return

    # grid setup (SdfBuilder::setupGrid through a tiny build)
    rows = []
    for name, kw in SETUP_CASES:
        v, t = ms[name]
        rows.append((name, kw, _spec_only(v, t, kw)))
    np.savez_compressed(
        os.path.join(HERE, "setup_grid.npz"),
        mesh=np.array([r[0] for r in rows]),
        padding=np.array([r[1]["padding"] for r in rows]),
        voxel_size=np.array([r[1]["voxel_size"] for r in rows]),
        target=np.array([r[1]["target_resolution"] for r in rows]),
        maxres=np.array([r[1]["max_resolution"] for r in rows]),
        shape=np.array([r[2]["shape"] for r in rows]),
        bmin=np.array([r[2]["bmin"] for r in rows]),
        bmax=np.array([r[2]["bmax"] for r in rows]),
        voxel=np.array([r[2]["voxel"] for r in rows]))

    # dense builds + queries
    for name, kw, n in [("cube", dict(target_resolution=16, max_resolution=16), 4000),
                        ("cyl", dict(target_resolution=24, max_resolution=32), 4000),
                        ("torus", dict(target_resolution=24, max_resolution=32), 4000)]:
        v, t = ms[name]
        g = ref.build_dense(v, t, padding=0.1, **kw)
        info = g.info()
        d = g.dense_arrays()
        pts = query_points(info, n, seed=11)
        np.savez_compressed(os.path.join(HERE, f"dense_{name}.npz"), verts=v, tris=t,
                            shape=np.array(info["shape"]), bmin=info["bmin"], bmax=info["bmax"],
                            voxel=info["voxel"], target=kw["target_resolution"],
                            maxres=kw["max_resolution"], pts=pts, **d, **ref_queries(g, pts))

    # sparse builds + queries
    for name, kw, n in [("cube", dict(target_resolution=32, max_resolution=32, band_voxels=3), 4000),
                        ("cyl", dict(target_resolution=48, max_resolution=64, band_voxels=2), 4000)]:
        v, t = ms[name]
        g = ref.build_sparse(v, t, padding=0.1, **kw)
        info = g.info()
        d = g.sparse_arrays()
        pts = query_points(info, n, seed=12)
        np.savez_compressed(os.path.join(HERE, f"sparse_{name}.npz"), verts=v, tris=t,
                            shape=np.array(info["shape"]), bmin=info["bmin"], bmax=info["bmax"],
                            voxel=info["voxel"], target=kw["target_resolution"],
                            maxres=kw["max_resolution"], band_voxels=kw["band_voxels"],
                            band=info["band"], block_dim=info["block_dim"], halo=info["halo"],
                            pts=pts, **d, **ref_queries(g, pts))

    # signed nearest (findSignedNearest) on meshes with ties and shared edges
    for name in ("torus", "gear", "cyl"):
        v, t = ms[name]
        rng = np.random.default_rng(13)
        lo, hi = v.min(0), v.max(0)
        ext = hi - lo
        pts = rng.uniform(lo - 0.2 * ext, hi + 0.2 * ext, (3000, 3))
        sd, cp, fn, tri = ref.signed_nearest(v, t, pts)
        np.savez_compressed(os.path.join(HERE, f"nearest_{name}.npz"), verts=v, tris=t, pts=pts,
                            sd=sd, cp=cp, fn=fn, tri=tri)

    # SDFO files written by the reference
    v, t = ms["cube"]
    ref.build_dense(v, t, padding=0.1, target_resolution=8, max_resolution=8).save(
        os.path.join(HERE, "cube8_dense.sdf"))
    ref.build_sparse(v, t, padding=0.1, target_resolution=16, max_resolution=16,
                     band_voxels=2).save(os.path.join(HERE, "cube16_sparse.sdf"))

    _prototype_fixtures(a.reference, ms)
    _contact_aware_fixtures(ms)
    _broadphase_fixtures(a.reference)
    _be_fixtures(a.reference)
    print("golden fixtures written to", HERE)


CA_CASES = [
    # (file, mesh, corner-normal kind, SdfBuilder::buildContactAware kwargs)
    ("ca_dense_cube", "cube", "face", dict(target_resolution=16, max_resolution=16)),
    ("ca_dense_torus", "torus", "smooth", dict(target_resolution=20, max_resolution=20,
                                               max_candidates=3)),
    ("ca_sparse_gear", "gear", "crease", dict(target_resolution=32, max_resolution=32, sparse=True,
                                              band_voxels=3)),
    ("ca_sparse_cube_notiles", "cube", "face", dict(target_resolution=16, max_resolution=16,
                                                    sparse=True, band_voxels=2,
                                                    use_tile_acceleration=False)),
]


def _contact_aware_fixtures(ms):
    """SdfBuilder::buildContactAware / buildSparseContactAware, queryFast in
    ContactAware mode with its candidate lists, contact-aware SDFO files and
    a NEXDYN_CONTACT_AWARE_SURFACE file parsed by the reference."""
    for fname, mesh, kind, kw in CA_CASES:
        v, t = ms[mesh]
        cn = M.corner_normals(v, t, kind)
        g = ref.build_contact_aware(v, t, cn, padding=0.1, **kw)
        info = g.info()
        ca = ref.ca_arrays(g)
        prim = g.sparse_arrays() if info["sparse"] else g.dense_arrays()
        pts = query_points(info, 3000, seed=14)
        q = ref.query_candidates(g, 4, pts)
        extra = {} if not info["sparse"] else dict(block_dim=info["block_dim"], halo=info["halo"],
                                                    band=info["band"])
        np.savez_compressed(
            os.path.join(HERE, f"{fname}.npz"), verts=v, tris=t, corner_normals=cn,
            params=np.array(repr(kw)), shape=np.array(info["shape"]), bmin=info["bmin"],
            bmax=info["bmax"], voxel=info["voxel"], stride=ca["stride"], count=ca["count"],
            cphi=ca["phi"], cnormal=ca["normal"], cbranch=ca["branch"], pts=pts,
            **{f"prim_{k}": val for k, val in prim.items() if val is not None},
            **{f"q_{k}": val for k, val in q.items()}, **extra)
    v, t = ms["cube"]
    cn = M.corner_normals(v, t, "face")
    ref.build_contact_aware(v, t, cn, padding=0.1, target_resolution=8, max_resolution=8).save(
        os.path.join(HERE, "ca_cube8_dense.sdf"))
    ref.build_contact_aware(v, t, cn, padding=0.1, target_resolution=16, max_resolution=16,
                            sparse=True, band_voxels=2).save(
        os.path.join(HERE, "ca_cube16_sparse.sdf"))
    v, t = M.torus(0.05, 0.01, 12, 6)
    path = os.path.join(HERE, "torus_small.ncas")
    M.write_ca_surface(path, v, t, M.corner_normals(v, t, "smooth"), name="ring")
    rv, rt, rcn = ref.load_ca_surface(path)
    np.savez_compressed(os.path.join(HERE, "torus_small_ncas.npz"), verts=rv, tris=rt,
                        corner_normals=rcn)


def _spec_only(v, t, kw):
    # the builder's GridSpec; a coarse copy of the mesh keeps this fast
    g = ref.build_dense(v, t, **kw) if np.prod(_raw_shape(v, kw)) <= 20_000_000 else None
    if g is None:
        raise RuntimeError("setup case too large")
    inf = g.info()
    return dict(shape=inf["shape"], bmin=inf["bmin"], bmax=inf["bmax"], voxel=inf["voxel"])


def _raw_shape(v, kw):
    vmin, vmax = v.min(0), v.max(0)
    diag = np.linalg.norm(vmax - vmin)
    size = (vmax - vmin) + 2 * kw["padding"] * diag
    h = kw["voxel_size"] if kw["voxel_size"] > 0 else size.max() / kw["target_resolution"]
    return np.minimum(np.ceil(size / h), kw["max_resolution"])


def _prototype_fixtures(reference, ms):
    proto = os.path.join(reference, "prototype")
    sys.path.insert(0, proto)
    from src.sdf_grid import TrilinearSDFGrid  # noqa: E402
    from src.dynamics.contacts_sdf import SDFContactEngine  # noqa: E402
    from src.geometry.quadrature import QuadratureMesh  # noqa: E402

    v, t = ms["cube"]
    g = ref.build_dense(v, t, padding=0.1, target_resolution=32, max_resolution=32)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "cube32.sdf")
        assert g.save(path)
        grid = TrilinearSDFGrid(path)
        info = g.info()
        rng = np.random.default_rng(21)
        pts = rng.uniform(info["bmin"] - 0.01, info["bmax"] + 0.01, (3000, 3))
        gq, raw, gn, unit, valid = grid.query_batch(pts)
        d = g.dense_arrays()

        # contact: torus quadrature on the cube SDF through SDFContactEngine.evaluate
        tv, tt = M.torus(0.05, 0.01, 48, 12)
        qx, qw = M.centroid_quadrature(tv, tt, normalize=False)
        poses = []
        res = []
        rng = np.random.default_rng(22)
        for _ in range(12):
            z = rng.uniform(0.058, 0.064)
            ax = rng.normal(size=3)
            ax[2] = 0.0
            ax /= np.linalg.norm(ax)
            ang = np.deg2rad(rng.uniform(0.0, 5.0))
            K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
            RA = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
            rA = np.array([rng.uniform(-1e-3, 1e-3), rng.uniform(-1e-3, 1e-3), z])
            vA = rng.normal(size=3) * 0.05
            wA = rng.normal(size=3) * 0.5
            qm = QuadratureMesh(qx.copy(), qw.copy())
            eng = SDFContactEngine()
            eng.register_pair(0, qm, grid, narrow_margin=1e9)
            model, state, cp = _mini_model(rA, RA, vA, wA)
            FA, tA, FB, tB = eng.evaluate(cp, state, model)
            poses.append(np.concatenate([rA, RA.ravel(), vA, wA]))
            res.append(np.concatenate([FA, tA, FB, tB]))
        np.savez_compressed(os.path.join(HERE, "prototype_cube32.npz"), phi=d["phi"],
                            normal=d["normal"], shape=np.array(info["shape"]), bmin=info["bmin"],
                            bmax=info["bmax"], voxel=info["voxel"], pts=pts, g=gq, raw_grad=raw,
                            grad_norm=gn, unit=unit, valid=valid, quad_x=qx, quad_w=qw,
                            poses=np.array(poses), forces=np.array(res),
                            k=1e9, order=2.0, damping=50.0, mu=0.3, reg=1e-4)


def _rot(axis, deg):
    ax = np.asarray(axis, float)
    ax = ax / np.linalg.norm(ax)
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    a = np.deg2rad(deg)
    return np.eye(3) + np.sin(a) * K + (1 - np.cos(a)) * K @ K


def _bvh_leaves(bvh):
    """The reference tree's leaves in the order AABB_BVH.query's stack visits
    them (bvh.py:71-80), with their boxes."""
    stack, order, boxes = [bvh.root], [], []
    while stack:
        node = stack.pop()
        if node.indices is not None:
            order.append(np.asarray(node.indices, np.int32))
            boxes.append(np.concatenate([node.aabb_min, node.aabb_max]))
        else:
            stack.append(node.left)
            stack.append(node.right)
    starts = np.concatenate([[0], np.cumsum([len(o) for o in order])]).astype(np.int32)
    return np.concatenate(order), starts, np.array(boxes)


def _broadphase_fixtures(reference):
    """AABB_BVH (geometry/bvh.py) over quadrature clouds and its query results,
    and SDFContactEngine.evaluate / measure_pair with the engine's default
    culling (register_pair narrow_margin 0.01) on a slab whose top face is the
    plane z = 0 of its SDF frame, body A a torus in many poses."""
    proto = os.path.join(reference, "prototype")
    if proto not in sys.path:
        sys.path.insert(0, proto)
    from src.dynamics.contacts_sdf import SDFContactEngine  # noqa: E402
    from src.geometry.bvh import AABB_BVH  # noqa: E402
    from src.geometry.quadrature import QuadratureMesh  # noqa: E402
    from src.sdf_grid import TrilinearSDFGrid  # noqa: E402

    rng = np.random.default_rng(31)
    tv, tt = M.torus(0.03, 0.008, 48, 12)
    qx, qw = M.centroid_quadrature(tv, tt, normalize=False)
    clouds = {"torus": qx, "random": rng.normal(size=(3000, 3)) * [0.05, 0.02, 0.01],
              "small": rng.uniform(-1, 1, (11, 3))}
    out = {}
    for name, X in clouds.items():
        bvh = AABB_BVH(X, leaf_size=16)
        order, starts, boxes = _bvh_leaves(bvh)
        lo0, hi0 = X.min(0), X.max(0)
        qmins, qmaxs, results = [], [], []
        for k in range(40):
            c = rng.uniform(lo0, hi0)
            h = rng.uniform(0.0, 0.6, 3) * (hi0 - lo0)
            qmin, qmax = c - h, c + h
            if k % 10 == 7:  # inverted on one axis, as rotated boxes give
                a = k % 3
                qmin[a], qmax[a] = qmax[a], qmin[a]
            if k % 10 == 9:  # enclosing everything
                qmin, qmax = lo0 - 1.0, hi0 + 1.0
            if k % 10 == 8:  # beside the cloud
                qmin, qmax = hi0 + 1.0, hi0 + 2.0
            res = bvh.query(qmin, qmax)
            qmins.append(qmin)
            qmaxs.append(qmax)
            results.append(np.asarray(res, np.int32))
        rs = np.concatenate([[0], np.cumsum([len(r) for r in results])]).astype(np.int32)
        out[name] = dict(points=X, order=order, starts=starts, boxes=boxes, qmin=np.array(qmins),
                         qmax=np.array(qmaxs), results=np.concatenate(results), result_starts=rs)
    np.savez_compressed(os.path.join(HERE, "point_bvh.npz"),
                        **{f"{c}_{k}": v for c, d in out.items() for k, v in d.items()})

    # the slab: 0.3 x 0.3 x 0.05, top face at z = 0
    cv, ct = M.cube(1.0)
    sv = cv * np.array([0.3, 0.3, 0.05]) + np.array([0.0, 0.0, -0.025])
    g = ref.build_dense(sv, ct, padding=0.1, target_resolution=32, max_resolution=32)
    info = g.info()
    d = g.dense_arrays()
    poses, bodyb, forces, meas = [], [], [], []
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "slab.sdf")
        assert g.save(path)
        grid = TrilinearSDFGrid(path)
        cases = []
        for _ in range(10):  # lying on the plane, small tilts
            cases.append((np.array([rng.uniform(-0.02, 0.02), rng.uniform(-0.02, 0.02),
                                    rng.uniform(0.0065, 0.0085)]),
                          _rot(rng.normal(size=3), rng.uniform(0, 6)), np.zeros(3), np.eye(3)))
        for deg in (30, 60, 90, 120, 150, 180):  # on edge / upside down
            R = _rot(rng.normal(size=3), deg)
            z = -(R @ qx.T)[2].min() - 0.0015
            cases.append((np.array([rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05), z]), R,
                          np.zeros(3), np.eye(3)))
        cases.append((np.array([0.6, 0.0, 0.007]), np.eye(3), np.zeros(3), np.eye(3)))  # far away
        cases.append((np.array([0.17, 0.0, 0.0075]), _rot([0, 1, 0], 10), np.zeros(3), np.eye(3)))
        cases.append((np.array([0.0, 0.0, 0.04]), np.eye(3), np.zeros(3), np.eye(3)))  # above
        for _ in range(4):  # body B moved and turned
            rB = rng.uniform(-0.02, 0.02, 3)
            RB = _rot([0, 0, 1], rng.uniform(-20, 20)) @ _rot(rng.normal(size=3), rng.uniform(0, 5))
            RA = RB @ _rot(rng.normal(size=3), rng.uniform(0, 8))
            rA = rB + RB @ np.array([rng.uniform(-0.03, 0.03), rng.uniform(-0.03, 0.03), 0.0075])
            cases.append((rA, RA, rB, RB))
        for rA, RA, rB, RB in cases:
            vA = rng.normal(size=3) * 0.05
            wA = rng.normal(size=3) * 0.5
            vB = rng.normal(size=3) * 0.01
            wB = rng.normal(size=3) * 0.1
            qm = QuadratureMesh(qx.copy(), qw.copy())
            eng = SDFContactEngine()
            eng.register_pair(0, qm, grid)
            model, state, cp = _mini_model(rA, RA, vA, wA, rB, RB, vB, wB)
            FA, tA, FB, tB = eng.evaluate(cp, state, model)
            m = eng.measure_pair(cp, state, model)
            poses.append(np.concatenate([rA, RA.ravel(), vA, wA]))
            bodyb.append(np.concatenate([rB, RB.ravel(), vB, wB]))
            forces.append(np.concatenate([FA, tA, FB, tB]))
            meas.append([m.gap, m.penetration, m.normal_velocity, m.min_point_index, m.active_count,
                         m.valid_count])
    np.savez_compressed(os.path.join(HERE, "engine_culling.npz"), phi=d["phi"], normal=d["normal"],
                        shape=np.array(info["shape"]), bmin=info["bmin"], bmax=info["bmax"],
                        voxel=info["voxel"], quad_x=qx, quad_w=qw, poses=np.array(poses),
                        body_b=np.array(bodyb), forces=np.array(forces), measure=np.array(meas),
                        k=1e9, order=2.0, damping=50.0, mu=0.3, reg=1e-4, narrow_margin=0.01)


BE_SCENES = [
    # name, torus tilt (axis, deg), start height of the lowest point above the
    # plane, v, w, mass, inertia diag, k, order, damping, mu, steps
    ("flat_drop", ([1, 0, 0], 0.0), 0.002, [0.03, 0.01, -0.15], [0.5, -0.3, 0.2], 0.05,
     [1.2e-5, 1.2e-5, 2.2e-5], 1e5, 1, 5.0, 0.3, 160),
    ("tilted_drop", ([1, 1, 0], 20.0), 0.0015, [0.0, 0.02, -0.1], [0.0, 0.4, -0.1], 0.05,
     [1.2e-5, 1.2e-5, 2.2e-5], 1e9, 2, 50.0, 0.3, 160),
]


def _be_fixtures(reference):
    """BackwardEulerIntegrator.step (prototype/src/integrators/implicit_be.py)
    run by the prototype itself: a torus (body A, centroid quadrature) dropped
    on the slab of _broadphase_fixtures (body B, fixed, TrilinearSDFGrid of
    the reference-built .sdf), SDFContactEngine with its default culling.
    implicit_be.py imports geometry/box_sdf.py, which the checkout does not
    ship; a stand-in module with an empty BoxSDF class is registered first
    (the integrator only tests isinstance against it in a helper the step
    does not call).  Every step records the full integrator state before and
    after it."""
    import types

    proto = os.path.join(reference, "prototype")
    if proto not in sys.path:
        sys.path.insert(0, proto)
    stub = types.ModuleType("src.geometry.box_sdf")

    class BoxSDF:  # noqa: D401 - stand-in for the missing module
        pass

    stub.BoxSDF = BoxSDF
    sys.modules["src.geometry.box_sdf"] = stub
    from src.dynamics.contacts_sdf import SDFContactEngine  # noqa: E402
    from src.dynamics.state import State  # noqa: E402
    from src.geometry.quadrature import QuadratureMesh  # noqa: E402
    from src.integrators.implicit_be import BackwardEulerIntegrator, ContactPhase  # noqa: E402
    from src.ir.body import RigidBody  # noqa: E402
    from src.ir.contact import ContactPair  # noqa: E402
    from src.ir.system_model import SystemModel  # noqa: E402
    from src.sdf_grid import TrilinearSDFGrid  # noqa: E402

    tv, tt = M.torus(0.03, 0.008, 48, 12)
    qx, qw = M.centroid_quadrature(tv, tt, normalize=False)
    cv, ct = M.cube(1.0)
    sv = cv * np.array([0.3, 0.3, 0.05]) + np.array([0.0, 0.0, -0.025])
    g = ref.build_dense(sv, ct, padding=0.1, target_resolution=32, max_resolution=32)
    info = g.info()
    d = g.dense_arrays()
    out = {}
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "slab.sdf")
        assert g.save(path)
        grid = TrilinearSDFGrid(path)
        for (name, (axis, deg), lift, v0, w0, mass, inert, k, order, damping, mu,
             nsteps) in BE_SCENES:
            RA = _rot(axis, deg) if deg else np.eye(3)
            z0 = -(RA @ qx.T)[2].min() + lift
            model = SystemModel()
            model.add_body(RigidBody("torus", 1, mass=mass, inertia_body=np.diag(inert),
                                     initial_r=np.array([0.0, 0.0, z0]), initial_R=RA,
                                     initial_v=np.array(v0, float), initial_omega=np.array(w0, float)))
            model.add_body(RigidBody("slab", 2, fixed=True))
            cp = ContactPair("c", 7, 1, 2, normal_stiffness=k, friction_coefficient=mu,
                             activation_distance=1e-5, k_order=order,
                             quadrature_settings={"damping": damping, "regularizer": 1e-4})
            model.add_contact(cp)
            eng = SDFContactEngine()
            eng.register_pair(cp.id, QuadratureMesh(qx.copy(), qw.copy()), grid)
            integ = BackwardEulerIntegrator(model, contact_engine=eng)
            state = State(model)
            i = state.body_idx(1)
            rows = []
            for _ in range(nsteps):
                st = integ._contact_states[cp.id]
                pre = np.concatenate([[state.t], state.r[i], state.R[i].ravel(), state.v[i],
                                      state.omega[i],
                                      [st.phase.value, st.dt_current, st.stable_count,
                                       st.release_count, st.min_dt_hits, st.last_gap,
                                       st.last_penetration, st.last_normal_velocity, st.last_toi]])
                h = integ.step(state, 1e-3)
                rows.append(np.concatenate([pre, [h]]))
            st = integ._contact_states[cp.id]
            last = np.concatenate([[state.t], state.r[i], state.R[i].ravel(), state.v[i],
                                   state.omega[i],
                                   [st.phase.value, st.dt_current, st.stable_count, st.release_count,
                                    st.min_dt_hits, st.last_gap, st.last_penetration,
                                    st.last_normal_velocity, st.last_toi], [0.0]])
            out[name] = np.array(rows + [last])
            out[name + "_params"] = np.array([mass, *inert, k, order, damping, mu, 1e-4])
            assert ContactPhase.ACTIVE.value == 3
    np.savez_compressed(os.path.join(HERE, "be_steps.npz"), phi=d["phi"], normal=d["normal"],
                        shape=np.array(info["shape"]), bmin=info["bmin"], bmax=info["bmax"],
                        voxel=info["voxel"], quad_x=qx, quad_w=qw, **out)


def _mini_model(rA, RA, vA, wA, rB=None, RB=None, vB=None, wB=None):
    """Minimal stand-ins for the IR model / state objects evaluate() reads:
    two bodies (A moving, B at the origin unless given), no markers."""
    rB = np.zeros(3) if rB is None else rB
    RB = np.eye(3) if RB is None else RB
    vB = np.zeros(3) if vB is None else vB
    wB = np.zeros(3) if wB is None else wB

    class Body:
        def __init__(self, i):
            self.id = i

    class Frames(dict):
        def get(self, k, default=None):
            return None

    class Model:
        bodies = {0: Body(0), 1: Body(1)}
        frames = Frames()

    class State:
        r = np.stack([rA, rB])
        R = np.stack([RA, RB])
        v = np.stack([vA, vB])
        omega = np.stack([wA, wB])

        @staticmethod
        def body_idx(i):
            return i

    class CP:
        id = 0
        body_a_id = 0
        body_b_id = 1
        normal_stiffness = 1e9
        friction_coefficient = 0.3
        activation_distance = 1e-5
        k_order = 2
        quadrature_settings = {"regularizer": 1e-4, "damping": 50.0}
        action_marker_id = None
        base_marker_id = None

    return Model(), State(), CP()


if __name__ == "__main__":
    main()
