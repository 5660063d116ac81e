"""GPU SDF construction against the oracle.

Reference-order mode (default) must reproduce the reference bit for bit:
FP64 signed distance, normal, witness point and Hessian of every voxel, the
sparse block set and its FP32 payload.  The FP32 query payload must be the
FP64 results rounded to float.  LBVH mode must agree on every distance and on
every sign the parity ray decides."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _meshes():
    from sdfo import meshes as M

    return {
        "cube": M.cube(0.1),
        "cyl": M.hollow_cylinder(0.05, 0.04, 0.02, n_az=64, n_vert=4),
        "torus": M.torus(0.05, 0.01, 48, 12),
        "gear": M.gear_prism(40, 0.05, 0.01, 20000),
        "one_triangle": (np.array([[0.0, 0, 0], [0.1, 0, 0], [0, 0.1, 0.02]]),
                         np.array([[0, 1, 2]], np.int32)),
        "open_quad": (np.array([[0.0, 0, 0], [0.1, 0, 0], [0.1, 0.1, 0], [0, 0.1, 0.0]]),
                      np.array([[0, 1, 2], [0, 2, 3]], np.int32)),
        "degenerate": (np.array([[0.0, 0, 0], [0.1, 0, 0], [0.05, 0.0, 0], [0.0, 0.1, 0.05],
                                 [0.0, 0.0, 0.1]]),
                       np.array([[0, 1, 2], [0, 1, 3], [1, 3, 4], [0, 4, 3], [0, 1, 4]], np.int32)),
    }


def _set_mode(mode):
    from sdfo import _native as N

    N.check(N.load().sdfo_set_bvh_mode(mode))


@pytest.mark.parametrize("name,res", [("cube", 32), ("cyl", 48), ("torus", 40), ("gear", 64),
                                      ("one_triangle", 16), ("open_quad", 16),
                                      ("degenerate", 24)])
def test_dense_build_bit_identical(cuda, port, name, res):
    from sdfo import SdfGrid

    _set_mode(0)
    v, t = _meshes()[name]
    P = port.build_dense(v, t, padding=0.1, target_resolution=res, max_resolution=res)
    g = SdfGrid.build_dense(v, t, padding=0.1, target_resolution=res, max_resolution=res)
    assert g.shape == tuple(P["spec"]["shape"])
    assert np.array_equal(g.bmin, P["spec"]["bmin"]) and np.array_equal(g.voxel, P["spec"]["voxel"])
    d = g.export_dense()
    assert np.array_equal(d["phi"], P["phi"])
    assert np.array_equal(d["normal"], P["normal"])
    assert np.array_equal(d["witness"], P["witness"])
    assert np.array_equal(d["hessian"], P["hessian"])
    pay = g.payload().cpu().numpy()
    assert np.array_equal(pay[:, 0], P["phi"].astype(np.float32))
    assert np.array_equal(pay[:, 1:], P["normal"].astype(np.float32))


@pytest.mark.parametrize("name", ["cube", "cyl", "torus"])
def test_dense_build_matches_reference_golden(cuda, name):
    from sdfo import SdfGrid

    _set_mode(0)
    gd = golden(f"dense_{name}.npz")
    g = SdfGrid.build_dense(gd["verts"], gd["tris"], padding=0.1,
                            target_resolution=int(gd["target"]), max_resolution=int(gd["maxres"]))
    d = g.export_dense()
    for k in ("phi", "normal", "witness", "hessian"):
        assert np.array_equal(d[k], gd[k]), k


def test_dense_build_c1_cube64(cuda, port):
    """BASELINE config 1 grid: cube 0.1 m at 64^3 with 4 voxels of padding."""
    from sdfo import SdfGrid
    from sdfo import workloads as W

    _set_mode(0)
    c = W.c1_cube64()
    g = SdfGrid.build_dense(c["verts"], c["tris"], **c["build"])
    assert g.shape == (64, 64, 64)
    P = port.build_dense(c["verts"], c["tris"], **c["build"])
    d = g.export_dense()
    assert np.array_equal(d["phi"], P["phi"])
    assert np.array_equal(d["normal"], P["normal"])
    # 4 voxels of padding: the cube face lies 4 voxels inside the grid boundary
    assert np.isclose((0.05 - g.bmax[0]) / g.voxel[0], -4.0, atol=1e-9)


@pytest.mark.parametrize("name,res,band", [("cube", 32, 3), ("cyl", 64, 2), ("gear", 64, 3),
                                           ("torus", 64, 3)])
def test_sparse_build_bit_identical(cuda, port, name, res, band):
    from sdfo import SdfGrid

    _set_mode(0)
    v, t = _meshes()[name]
    P = port.build_sparse(v, t, padding=0.1, target_resolution=res, max_resolution=res,
                          band_voxels=band)
    g = SdfGrid.build_sparse(v, t, padding=0.1, target_resolution=res, max_resolution=res,
                             band_voxels=band)
    assert g.band_distance == P["band"]
    d = g.export_sparse()
    assert np.array_equal(d["ijk"], P["ijk"]), "sparse occupancy"
    assert np.array_equal(d["phi"], P["phi"])
    assert np.array_equal(d["normal"], P["normal"])
    assert np.array_equal(d["hessian"], P["hessian"])


@pytest.mark.parametrize("name", ["cube", "cyl"])
def test_sparse_build_matches_reference_golden(cuda, name):
    from sdfo import SdfGrid

    _set_mode(0)
    gd = golden(f"sparse_{name}.npz")
    g = SdfGrid.build_sparse(gd["verts"], gd["tris"], padding=0.1,
                             target_resolution=int(gd["target"]), max_resolution=int(gd["maxres"]),
                             band_voxels=int(gd["band_voxels"]))
    d = g.export_sparse()
    for k in ("ijk", "phi", "normal", "hessian"):
        assert np.array_equal(d[k], gd[k]), k


def test_c2_cylinder_dense_and_sparse(cuda, port):
    """BASELINE config 2 grids at full size: 128x128x64 dense (1M voxels) and
    the band-3 sparse grid, bit-identical to the oracle."""
    from sdfo import SdfGrid
    from sdfo import workloads as W

    _set_mode(0)
    c = W.c2_cylinder()
    g = SdfGrid.build_dense(c["verts"], c["tris"], **c["dense"])
    assert g.shape == (128, 128, 64)
    P = port.build_dense(c["verts"], c["tris"], **c["dense"])
    d = g.export_dense()
    assert np.array_equal(d["phi"], P["phi"])
    assert np.array_equal(d["normal"], P["normal"])
    gs = SdfGrid.build_sparse(c["verts"], c["tris"], **c["sparse"])
    Ps = port.build_sparse(c["verts"], c["tris"], **c["sparse"])
    ds = gs.export_sparse()
    assert np.array_equal(ds["ijk"], Ps["ijk"])
    assert np.array_equal(ds["phi"], Ps["phi"])
    assert np.array_equal(ds["normal"], Ps["normal"])


@pytest.mark.parametrize("name", ["cyl", "torus", "gear"])
def test_lbvh_mode_distances(cuda, port, name):
    """LBVH traversal: identical distances; identical signs wherever the parity
    ray hits the mesh (the only tie-dependent sign is the 0-hit fallback)."""
    from sdfo import SdfGrid

    v, t = _meshes()[name]
    P = port.build_dense(v, t, padding=0.1, target_resolution=40, max_resolution=40)
    _set_mode(1)
    try:
        g = SdfGrid.build_dense(v, t, padding=0.1, target_resolution=40, max_resolution=40)
    finally:
        _set_mode(0)
    d = g.export_dense()
    assert np.array_equal(np.abs(d["phi"]), np.abs(P["phi"]))
    b = port.Bvh(v, t)
    spec = P["spec"]
    nx, ny, nz = spec["shape"]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    c = spec["bmin"] + spec["voxel"] * (np.stack([i.ravel(), j.ravel(), k.ravel()], 1) + 0.5)
    hits = b.signed_nearest(c)["hits"]
    decided = hits > 0
    assert np.array_equal(np.signbit(d["phi"][decided]), np.signbit(P["phi"][decided]))


@pytest.mark.parametrize("name,res", [("cube", 32), ("cyl", 48), ("torus", 40), ("gear", 64)])
def test_traversal_counts_match_reference_order(cuda, port, name, res):
    """The dense fill's traversal work counted on the device
    (sdfo_build_traversal_stats) equals the oracle's recursive KdTree
    traversal count for count: nodes entered past the nearest search's cut,
    closest-point tests, ray-box tests and ray-triangle tests.  Equal totals
    over every voxel follow from the same visit order and the same cuts."""
    from sdfo import SdfGrid

    _set_mode(0)
    v, t = _meshes()[name]
    st = SdfGrid.traversal_stats(v, t, padding=0.1, target_resolution=res, max_resolution=res)
    spec = port.setup_grid(v, padding=0.1, target_resolution=res, max_resolution=res)
    nx, ny, nz = spec["shape"]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    idx = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    centres = spec["bmin"][None, :] + spec["voxel"][None, :] * (idx + 0.5)
    ref = port.Bvh(v, t).traversal_counts(centres)
    n = nx * ny * nz
    assert st["voxels"] == n
    assert np.array_equal(np.array(st["totals"], np.int64), ref), (st["totals"], ref)


def test_device_cache_reuse(cuda):
    """Freed grid storage is cached and reused: a second identical build
    gives identical data, the cache holds the freed blocks, and a zero limit
    releases them."""
    import ctypes

    from sdfo import SdfGrid
    from sdfo import _native as N

    lib = N.load()
    held = ctypes.c_int64(-1)
    try:
        N.check(lib.sdfo_device_cache(1 << 30, ctypes.byref(held)))
        v, t = _meshes()["torus"]
        a = SdfGrid.build_dense(v, t, target_resolution=40, max_resolution=40)
        ea = a.export_dense()
        a.close()
        N.check(lib.sdfo_device_cache(-1, ctypes.byref(held)))
        assert held.value > 0
        b = SdfGrid.build_dense(v, t, target_resolution=40, max_resolution=40)
        eb = b.export_dense()
        for k in ("phi", "normal", "witness", "hessian"):
            assert np.array_equal(ea[k], eb[k]), k
        b.close()
        N.check(lib.sdfo_device_cache(0, ctypes.byref(held)))
        assert held.value == 0
    finally:
        N.check(lib.sdfo_device_cache(1 << 30, None))


def test_empty_mesh_raises(cuda):
    from sdfo import SdfGrid, SdfoError

    with pytest.raises(SdfoError, match="Empty mesh provided to SdfBuilder"):
        SdfGrid.build_dense(np.zeros((0, 3)), np.zeros((0, 3), np.int32))


def test_build_stats(cuda):
    from sdfo import SdfGrid

    v, t = _meshes()["torus"]
    g = SdfGrid.build_dense(v, t, target_resolution=32, max_resolution=32)
    s = g.build_stats()
    assert s["voxels_filled"] == np.prod(g.shape)
    assert s["triangles"] == len(t) and s["bvh_nodes"] > 0


@pytest.mark.parametrize("tile", [(2, 2), (4, 2), (2, 3), (4, 1), (5, 3)])
def test_dense_fill_tile_shapes_bit_identical(cuda, port, tile):
    """Every voxel tile of the dense fill CTAs (a tuning knob) builds the
    oracle's grid bit for bit, with the same device-counted traversal work."""
    from sdfo import SdfGrid
    from sdfo import _native as N

    _set_mode(0)
    before = N.get_tuning()
    v, t = _meshes()["gear"]
    P = port.build_dense(v, t, padding=0.1, target_resolution=64, max_resolution=64)
    base = SdfGrid.traversal_stats(v, t, padding=0.1, target_resolution=64, max_resolution=64)
    try:
        N.set_tuning(fill_tile_log2_x=tile[0], fill_tile_log2_y=tile[1])
        g = SdfGrid.build_dense(v, t, padding=0.1, target_resolution=64, max_resolution=64)
        d = g.export_dense()
        for k in ("phi", "normal", "witness", "hessian"):
            assert np.array_equal(d[k], P[k]), k
        st = SdfGrid.traversal_stats(v, t, padding=0.1, target_resolution=64, max_resolution=64)
        assert st["totals"] == base["totals"]
    finally:
        N.set_tuning(**before)


@pytest.mark.parametrize("name,res", [("gear", 64), ("torus", 40), ("one_triangle", 16),
                                      ("degenerate", 24)])
def test_lbvh_stackless_equals_stack(cuda, name, res):
    """The stackless LBVH traversals (parent links) give the stack
    traversals' grid bit for bit, dense and sparse, with the same
    device-counted work."""
    from sdfo import SdfGrid
    from sdfo import _native as N

    v, t = _meshes()[name]
    kw = dict(padding=0.1, target_resolution=res, max_resolution=res)
    before = N.get_tuning()
    out = {}
    try:
        _set_mode(1)
        for mode in (1, 2):
            N.set_tuning(lbvh_traversal=mode)
            d = SdfGrid.build_dense(v, t, **kw).export_dense()
            sp = SdfGrid.build_sparse(v, t, band_voxels=3, **kw).export_sparse()
            st = SdfGrid.traversal_stats(v, t, **kw)["totals"]
            out[mode] = (d, sp, st)
    finally:
        _set_mode(0)
        N.set_tuning(**before)
    (d1, s1, c1), (d2, s2, c2) = out[1], out[2]
    for k in ("phi", "normal", "witness", "hessian"):
        assert np.array_equal(d1[k], d2[k]), k
    for k in ("ijk", "phi", "normal"):
        assert np.array_equal(s1[k], s2[k]), k
    assert c1 == c2


def test_triangle_cull_off_equals_on(cuda, port):
    """The FP32 triangle-box cull only skips closest-point tests that cannot
    replace the best: with it off (a tuning knob) the grid is the same bit
    for bit, and the device counts more FP64 tests."""
    from sdfo import SdfGrid
    from sdfo import _native as N

    _set_mode(0)
    v, t = _meshes()["gear"]
    kw = dict(padding=0.1, target_resolution=64, max_resolution=64)
    before = N.get_tuning()
    out = {}
    try:
        for cull in (1, 2):
            N.set_tuning(triangle_cull=cull)
            out[cull] = (SdfGrid.build_dense(v, t, **kw).export_dense(),
                         SdfGrid.build_sparse(v, t, band_voxels=3, **kw).export_sparse(),
                         SdfGrid.traversal_stats(v, t, **kw))
    finally:
        N.set_tuning(**before)
    for k in ("phi", "normal", "witness", "hessian"):
        assert np.array_equal(out[1][0][k], out[2][0][k]), k
    for k in ("ijk", "phi", "normal", "hessian"):
        assert np.array_equal(out[1][1][k], out[2][1][k]), k
    on, off = out[1][2], out[2][2]
    assert on["totals"] == off["totals"]
    assert off["exact_triangle_tests_per_voxel"] == off["nearest_triangle_tests_per_voxel"]
    assert on["exact_triangle_tests_per_voxel"] < off["exact_triangle_tests_per_voxel"]
