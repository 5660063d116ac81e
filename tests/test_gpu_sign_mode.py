"""SDFO_SIGN_PSEUDONORMAL builds (no reference counterpart) against the
pseudo-normal oracle (oracle/pseudo_normal.py) on closed, consistently
oriented meshes, dense and sparse:
* every voxel's sign equals the oracle's, and every |phi| equals the
  reference-mode build bit for bit (the distance search is unchanged);
* the LBVH build (lowest index at exact ties) gives the same signs as the
  reference-order build: the pseudo-normal sign does not depend on which of
  several equidistant triangles is kept;
* against the reference's ray parity, a voxel may differ only where the
  parity ray hits nothing (the point is outside) and the reference's
  fallback -- the face normal of the nearest triangle -- reports inside,
  which happens at concave vertices and edges (the gear's tooth roots);
  there the pseudo-normal reports outside.  Elsewhere normals are equal."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _meshes():
    from sdfo import meshes as M

    return {"torus": (M.torus(0.05, 0.01, 48, 12), 40), "cyl": (M.hollow_cylinder(0.05, 0.04, 0.02, n_az=64,
                                                                                    n_vert=4), 48),
            "cube": (M.cube(0.1), 32), "gear": (M.gear_prism(24, 0.05, 0.01, 3000), 32)}


def _centres(spec):
    sh = spec["shape"]
    k, j, i = np.meshgrid(np.arange(sh[2]), np.arange(sh[1]), np.arange(sh[0]), indexing="ij")
    c = np.stack([i.ravel(), j.ravel(), k.ravel()], 1)  # x fastest
    return np.asarray(spec["bmin"]) + np.asarray(spec["voxel"]) * (c + 0.5)


def _modes(bvh, sign):
    from sdfo import _native as N

    N.check(N.load().sdfo_set_bvh_mode(bvh))
    N.check(N.load().sdfo_set_sign_mode(sign))


@pytest.mark.parametrize("name", ["torus", "cyl", "cube", "gear"])
def test_pseudonormal_dense_build(cuda, port, name):
    from oracle import pseudo_normal as PN

    from sdfo import SdfGrid

    (v, t), res = _meshes()[name]
    kw = dict(padding=0.1, target_resolution=res, max_resolution=res)
    try:
        _modes(0, 0)
        ref = SdfGrid.build_dense(v, t, **kw).export_dense()
        _modes(0, 1)
        g = SdfGrid.build_dense(v, t, **kw)
        d = g.export_dense()
        _modes(1, 1)
        dl = SdfGrid.build_dense(v, t, **kw).export_dense()
    finally:
        _modes(0, 0)
    spec = dict(bmin=g.bmin, voxel=g.voxel, shape=g.shape)
    ctr = _centres(spec)
    sd, _, _ = PN.signed_distance(v, t, ctr)
    assert np.array_equal(np.abs(d["phi"]), np.abs(ref["phi"]))
    assert np.array_equal(np.abs(sd), np.abs(d["phi"]))
    assert np.array_equal(np.sign(d["phi"]), np.sign(sd))
    # tie-independent: the LBVH build's signs and distances are the same
    assert np.array_equal(dl["phi"], d["phi"])
    # where the sign differs from the reference's ray parity
    flip = np.sign(d["phi"]) != np.sign(ref["phi"])
    assert np.array_equal(d["normal"][~flip], ref["normal"][~flip])
    if flip.any():
        hits = port.Bvh(v, t).signed_nearest(ctr[flip])["hits"]
        assert np.all(hits == 0) and np.all(ref["phi"][flip] < 0) and np.all(d["phi"][flip] > 0)


@pytest.mark.parametrize("name", ["torus", "gear"])
def test_pseudonormal_sparse_build(cuda, port, name):
    from oracle import pseudo_normal as PN

    from sdfo import SdfGrid

    (v, t), res = _meshes()[name]
    kw = dict(padding=0.1, target_resolution=res, max_resolution=res, band_voxels=3)
    try:
        _modes(0, 0)
        ref = SdfGrid.build_sparse(v, t, **kw).export_sparse()
        _modes(0, 1)
        g = SdfGrid.build_sparse(v, t, **kw)
        d = g.export_sparse()
    finally:
        _modes(0, 0)
    assert np.array_equal(d["ijk"], ref["ijk"])
    assert np.array_equal(np.abs(d["phi"]), np.abs(ref["phi"]))
    bd = 8
    lo = np.stack(np.meshgrid(np.arange(bd), np.arange(bd), np.arange(bd), indexing="ij"), -1)
    local = lo.transpose(2, 1, 0, 3).reshape(-1, 3)  # x fastest within a brick
    ijk = d["ijk"][:, None, :] * bd + local[None]
    inside = np.all(ijk < np.asarray(g.shape), axis=-1)
    ctr = np.asarray(g.bmin) + np.asarray(g.voxel) * (ijk + 0.5)
    sd, _, _ = PN.signed_distance(v, t, ctr[inside])
    assert np.array_equal(np.sign(d["phi"][inside]), np.sign(sd.astype(np.float32)))
