"""The oracle restatement (oracle/sdfo_port.cpp, oracle/contact_port.py) against
golden vectors produced by the reference itself (tests/golden/make_golden.py).

These pin the checker the CUDA kernels are compared with: grid setup, signed
distance, sign, normal, witness point, Hessian, sparse occupancy and every
query mode must reproduce the reference bit for bit (the restatement uses the
reference's own triangle tree, so even exactly equidistant triangles resolve
the same way)."""
import numpy as np
import pytest

from conftest import golden


def test_setup_grid_matches_reference(port):
    g = golden("setup_grid.npz")
    from sdfo import meshes as M

    ms = {"cube": M.cube(0.1), "cyl": M.hollow_cylinder(0.05, 0.04, 0.02, n_az=64, n_vert=4),
          "torus": M.torus(0.05, 0.01, 48, 12), "gear": M.gear_prism(24, 0.05, 0.01, 3000)}
    for i, name in enumerate(g["mesh"]):
        v, _ = ms[str(name)]
        s = port.setup_grid(v, float(g["padding"][i]), float(g["voxel_size"][i]),
                            int(g["target"][i]), int(g["maxres"][i]))
        assert tuple(s["shape"]) == tuple(g["shape"][i])
        assert np.array_equal(s["bmin"], g["bmin"][i])
        assert np.array_equal(s["bmax"], g["bmax"][i])
        assert np.array_equal(s["voxel"], g["voxel"][i])


def test_snap_resolution_ladder(port):
    # snapToStandardResolution (GridSpec.h:65-74)
    assert port.snap_resolution(1, 512) == 8
    assert port.snap_resolution(9, 512) == 16
    assert port.snap_resolution(49, 128) == 64
    assert port.snap_resolution(129, 128) == 128
    assert port.snap_resolution(100, 96) == 96
    assert port.snap_resolution(3000, 4096) == 4096  # falls through the ladder to maxRes


@pytest.mark.parametrize("name", ["cube", "cyl", "torus"])
def test_dense_build_matches_reference(port, name):
    g = golden(f"dense_{name}.npz")
    P = port.build_dense(g["verts"], g["tris"], padding=0.1,
                         target_resolution=int(g["target"]), max_resolution=int(g["maxres"]))
    assert tuple(P["spec"]["shape"]) == tuple(g["shape"])
    assert np.array_equal(P["phi"], g["phi"]), "signed distance must be bit-identical"
    assert np.array_equal(np.signbit(P["phi"]), np.signbit(g["phi"]))
    assert np.array_equal(P["normal"], g["normal"])
    assert np.array_equal(P["witness"], g["witness"])
    assert np.array_equal(P["hessian"], g["hessian"])
    # Hessian from the reference's own normals is bit-identical
    H = port.dense_hessian(P["spec"], g["normal"])
    assert np.array_equal(H, g["hessian"])


@pytest.mark.parametrize("name", ["cube", "cyl", "torus"])
def test_dense_queries_match_reference(port, name):
    g = golden(f"dense_{name}.npz")
    spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"],
                         shape=tuple(g["shape"]))
    for mode in range(4):
        q = port.query_dense(spec, g["phi"], g["normal"], g["hessian"], mode, g["pts"])
        assert np.array_equal(q["valid"], g[f"q{mode}_valid"])
        np.testing.assert_allclose(q["gap"], g[f"q{mode}_gap"], rtol=1e-13, atol=1e-16)
        np.testing.assert_allclose(q["unit"], g[f"q{mode}_normal"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(q["witness"], g[f"q{mode}_witness"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", ["cube", "cyl"])
def test_sparse_build_matches_reference(port, name):
    g = golden(f"sparse_{name}.npz")
    P = port.build_sparse(g["verts"], g["tris"], padding=0.1,
                          target_resolution=int(g["target"]), max_resolution=int(g["maxres"]),
                          band_voxels=int(g["band_voxels"]))
    assert P["band"] == float(g["band"])
    assert np.array_equal(P["ijk"], g["ijk"]), "sparse occupancy must match exactly"
    assert np.array_equal(P["phi"], g["phi"])
    assert np.array_equal(P["normal"], g["normal"])
    assert np.array_equal(P["hessian"], g["hessian"])
    H = port.sparse_hessian(P["spec"], int(g["block_dim"]), g["ijk"], g["normal"])
    assert np.array_equal(H, g["hessian"])


@pytest.mark.parametrize("name", ["cube", "cyl"])
def test_sparse_queries_match_reference(port, name):
    g = golden(f"sparse_{name}.npz")
    spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"],
                         shape=tuple(g["shape"]))
    for mode in range(4):
        q = port.query_sparse(spec, int(g["block_dim"]), g["ijk"], g["phi"], g["normal"],
                              g["hessian"], mode, g["pts"])
        assert np.array_equal(q["valid"], g[f"q{mode}_valid"])
        np.testing.assert_allclose(q["gap"], g[f"q{mode}_gap"], rtol=1e-13, atol=1e-16)
        np.testing.assert_allclose(q["unit"], g[f"q{mode}_normal"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("name", ["torus", "gear", "cyl"])
def test_signed_nearest_matches_reference(port, name):
    g = golden(f"nearest_{name}.npz")
    b = port.Bvh(g["verts"], g["tris"])
    r = b.signed_nearest(g["pts"])
    assert np.array_equal(r["sd"], g["sd"])
    assert np.array_equal(r["tri"], g["tri"])
    assert np.array_equal(r["cp"], g["cp"])
    assert np.array_equal(r["fn"], g["fn"])


def test_prototype_trilinear_matches_restatement(port):
    """TrilinearSDFGrid.query_batch (prototype/src/sdf_grid.py:138-204) vs the
    C++-order restatement on the same FP64 grid: equal to rounding."""
    g = golden("prototype_cube32.npz")
    spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"],
                         shape=tuple(g["shape"]))
    q = port.query_dense(spec, g["phi"], g["normal"], None, port.TRILINEAR, g["pts"])
    assert np.array_equal(q["valid"], g["valid"])
    v = g["valid"]
    np.testing.assert_allclose(q["gap"][v], g["g"][v], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(q["grad"][v], g["raw_grad"][v], rtol=1e-10, atol=1e-12)


def test_contact_restatement_matches_prototype(port):
    """oracle/contact_port.evaluate_pose vs SDFContactEngine.evaluate."""
    from oracle import contact_port as cp

    g = golden("prototype_cube32.npz")
    spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"],
                         shape=tuple(g["shape"]))

    def qb(Y):
        q = port.query_dense(spec, g["phi"], g["normal"], None, port.TRILINEAR, Y)
        gn = np.linalg.norm(q["grad"], axis=1)
        return q["gap"], q["grad"], gn, None, q["valid"]

    w = g["quad_w"] / g["quad_w"].sum()
    prm = dict(k=float(g["k"]), order=float(g["order"]), damping=float(g["damping"]),
               mu=float(g["mu"]), regularizer=float(g["reg"]))
    nonzero = 0
    for pose, ref_f in zip(g["poses"], g["forces"]):
        rA, RA, vA, wA = pose[:3], pose[3:12].reshape(3, 3), pose[12:15], pose[15:18]
        F, tau, _, _ = cp.evaluate_pose(qb, g["quad_x"], w, rA, RA, vA, wA, np.zeros(3),
                                        np.eye(3), np.zeros(3), np.zeros(3), **prm)
        scale = max(np.abs(ref_f[:6]).max(), 1e-12)
        assert np.abs(F - ref_f[:3]).max() <= 1e-9 * scale
        assert np.abs(tau - ref_f[3:6]).max() <= 1e-9 * scale
        nonzero += np.abs(ref_f[:3]).max() > 0
    assert nonzero >= 3, "fixture must contain poses in contact"
