"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a container where the reference checkout is present:

    make -C oracle ref port
    python tests/golden/make_golden.py [--reference /root/reference]

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
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", choices=["all", "contact_aware"], default="all")
    a = ap.parse_args()
    ms = meshes()
    if a.only == "contact_aware":
        _contact_aware_fixtures(ms)
        print("contact-aware fixtures written to", HERE)
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


def _mini_model(rA, RA, vA, wA):
    """Minimal stand-ins for the IR model / state objects evaluate() reads:
    two bodies (A moving, B fixed at the origin), no markers."""

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
        r = np.stack([rA, np.zeros(3)])
        R = np.stack([RA, np.eye(3)])
        v = np.stack([vA, np.zeros(3)])
        omega = np.stack([wA, np.zeros(3)])

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
