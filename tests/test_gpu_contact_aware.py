"""Contact-aware builds and ContactAware queries on the GPU against
fixtures made by the reference (SdfBuilder::buildContactAware /
buildSparseContactAware, queryFast; tests/golden/make_golden.py).

Builds: candidate counts, candidate phi / normal / branch ids and the
primary phi / normal / witness / Hessian bit-identical.  Queries: valid
flags, candidate counts and branch ids exact; gaps, normals and witnesses
are the reference's FP64 values rounded to FP32 (bound 2^-24 relative, 1e-6
of max(|value|, h) asserted)."""
import ast
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

pytestmark = pytest.mark.gpu

CASES = ["ca_dense_cube", "ca_dense_torus", "ca_sparse_gear", "ca_sparse_cube_notiles"]


def _gpu_build(g, bvh=0):
    from sdfo import SdfGrid
    from sdfo import _native as N

    N.check(N.load().sdfo_set_bvh_mode(bvh))
    try:
        return SdfGrid.build_contact_aware(g["verts"], g["tris"], g["corner_normals"], padding=0.1,
                                           **ast.literal_eval(str(g["params"])))
    finally:
        N.check(N.load().sdfo_set_bvh_mode(0))


@pytest.mark.parametrize("name", CASES)
def test_gpu_contact_aware_build_bit_identical(cuda, name):
    g = golden(f"{name}.npz")
    grid = _gpu_build(g)
    assert grid.shape == tuple(g["shape"])
    assert grid.candidate_stride == int(g["stride"])
    c = grid.export_candidates()
    s = int(g["stride"])
    assert np.array_equal(c["count"], g["count"].reshape(-1))
    assert np.array_equal(c["phi"], np.asarray(g["cphi"], np.float64).reshape(-1, s))
    assert np.array_equal(c["normal"], np.asarray(g["cnormal"], np.float64).reshape(-1, s, 3))
    assert np.array_equal(c["branch"], g["cbranch"].reshape(-1, s))
    if grid.is_sparse:
        d = grid.export_sparse()
        for k in ("ijk", "phi", "normal", "hessian"):
            assert np.array_equal(d[k], g[f"prim_{k}"]), k
    else:
        d = grid.export_dense()
        for k in ("phi", "normal", "witness", "hessian"):
            assert np.array_equal(d[k], g[f"prim_{k}"]), k


def _check_query(out, g, h):
    v = g["q_valid"].astype(bool)
    assert np.array_equal(out["valid"].astype(bool), v)
    assert np.array_equal(out["ncand"][v], g["q_ncand"][v])
    for k in ("gap", "normal", "witness"):
        ref = g[f"q_{k}"][v]
        got = out[k][v].astype(np.float64)
        assert np.all(np.abs(got - ref) <= 1e-6 * np.maximum(np.abs(ref), h)), k
    m = np.arange(8)[None, :] < g["q_ncand"][:, None]
    assert np.array_equal(out["kbranch"][m], g["q_kbranch"][m])
    for k in ("kgap", "knormal", "kwitness"):
        ref = g[f"q_{k}"][m]
        got = out[k][m].astype(np.float64)
        assert np.all(np.abs(got - ref) <= 1e-6 * np.maximum(np.abs(ref), h)), k


@pytest.mark.parametrize("name", CASES)
def test_gpu_contact_aware_queries_match_reference(cuda, name):
    import torch

    g = golden(f"{name}.npz")
    grid = _gpu_build(g)
    x = torch.tensor(g["pts"].astype(np.float32), device="cuda")
    out = {k: t.cpu().numpy() for k, t in grid.query_candidates(x, mode=4).items()}
    _check_query(out, g, float(g["voxel"][0]))
    # the plain query entry point in ContactAware mode gives the same result
    q = grid.query_tensors(x, mode=4, unit=True, witness=True, valid=True)
    assert np.array_equal(q["valid"].cpu().numpy(), out["valid"])
    assert np.array_equal(q["gap"].cpu().numpy(), out["gap"])
    assert np.array_equal(q["unit"].cpu().numpy(), out["normal"])
    assert np.array_equal(q["witness"].cpu().numpy(), out["witness"])


def test_host_buffer_candidates_match_device(cuda):
    import ctypes

    import torch

    from sdfo import _native as N

    g = golden("ca_sparse_gear.npz")
    grid = _gpu_build(g)
    pts = np.ascontiguousarray(g["pts"])
    n = len(pts)
    out = dict(gap=np.zeros(n, np.float32), normal=np.zeros((n, 3), np.float32),
               witness=np.zeros((n, 3), np.float32), valid=np.zeros(n, np.uint8),
               ncand=np.zeros(n, np.int32), kgap=np.zeros((n, 8), np.float32),
               knormal=np.zeros((n, 8, 3), np.float32), kwitness=np.zeros((n, 8, 3), np.float32),
               kbranch=np.zeros((n, 8), np.int32))
    P = [ctypes.c_void_p(out[k].ctypes.data) for k in ("gap", "normal", "witness", "valid", "ncand",
                                                         "kgap", "knormal", "kwitness", "kbranch")]
    N.check(N.load().sdfo_query_candidates_host(grid.handle, 4, ctypes.c_void_p(pts.ctypes.data), 1,
                                                n, *P, None))
    _check_query(out, g, float(g["voxel"][0]))
    dev = grid.query_candidates(torch.tensor(pts.astype(np.float32), device="cuda"), mode=4)
    assert np.array_equal(dev["kbranch"].cpu().numpy(), out["kbranch"])


@pytest.mark.parametrize("mode", [0, 2, 3])
def test_candidates_of_plain_modes(cuda, mode):
    """Modes without candidates report one candidate: the query's own result
    with branch id 0 (fastFromQueryResult)."""
    import torch

    g = golden("ca_dense_torus.npz")
    grid = _gpu_build(g)
    x = torch.tensor(g["pts"].astype(np.float32), device="cuda")
    c = grid.query_candidates(x, mode=mode)
    q = grid.query_tensors(x, mode=mode, unit=True, witness=True, valid=True)
    v = q["valid"].bool()
    assert torch.equal(c["valid"], q["valid"])
    assert torch.equal(c["ncand"], v.int())
    assert torch.equal(c["kgap"][v, 0], q["gap"][v])
    assert torch.equal(c["knormal"][v, 0], q["unit"][v])
    assert torch.all(c["kbranch"][v, 0] == 0) and torch.all(c["kbranch"][:, 1:] == -1)


def test_contact_aware_files_on_the_gpu(cuda, tmp_path):
    """A contact-aware SDFO file written by the reference loads onto the GPU
    (candidates attached) and answers like the grid built on the GPU; the GPU
    grid saves to the reference's bytes."""
    import torch

    from sdfo import SdfGrid
    from sdfo import meshes as M

    v, t = M.cube(0.1)
    cn = M.corner_normals(v, t, "face")
    built = SdfGrid.build_contact_aware(v, t, cn, padding=0.1, target_resolution=8,
                                        max_resolution=8)
    out = tmp_path / "cube8.sdf"
    assert built.save(str(out))
    assert out.read_bytes() == open(os.path.join(GOLDEN, "ca_cube8_dense.sdf"), "rb").read()
    loaded = SdfGrid.load(os.path.join(GOLDEN, "ca_cube8_dense.sdf"), mode=4)
    assert loaded.candidate_stride == 4
    rng = np.random.default_rng(3)
    x = torch.tensor(rng.uniform(-0.07, 0.07, (2000, 3)).astype(np.float32), device="cuda")
    a = built.query_candidates(x, mode=4)
    b = loaded.query_candidates(x, mode=4)
    for k in a:
        assert torch.equal(a[k], b[k]), k
    sparse = SdfGrid.build_contact_aware(v, t, cn, padding=0.1, target_resolution=16,
                                         max_resolution=16, sparse=True, band_voxels=2)
    out = tmp_path / "cube16.sdf"
    assert sparse.save(str(out))
    assert out.read_bytes() == open(os.path.join(GOLDEN, "ca_cube16_sparse.sdf"), "rb").read()
    ls = SdfGrid.load(os.path.join(GOLDEN, "ca_cube16_sparse.sdf"), mode=4)
    a = sparse.query_candidates(x, mode=4)
    b = ls.query_candidates(x, mode=4)
    for k in a:
        assert torch.equal(a[k], b[k]), k


def test_lbvh_mode_contact_aware(cuda):
    """The tile lists decide every candidate; the tree only answers voxels
    with an empty list, so the LBVH build agrees on a smooth torus."""
    g = golden("ca_dense_torus.npz")
    a = _gpu_build(g, bvh=0).export_candidates()
    b = _gpu_build(g, bvh=1).export_candidates()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("name", ["ca_dense_torus", "ca_sparse_gear"])
def test_contact_aware_walk_bit_identical(cuda, name):
    """The persistent walk kernel for ContactAware queries of float32 points
    on sparse grids (the default there; sdfo_tuning.query_walk) gives every
    output and candidate list bit for bit as the one-CTA-per-tile kernel
    does, for batches below one tile, between tiles and above the resident
    CTA count; dense grids take the per-tile kernel either way."""
    import torch

    from sdfo import _native as N

    g = golden(f"{name}.npz")
    grid = _gpu_build(g)
    rng = np.random.default_rng(12)
    lo, hi = np.array(grid.bmin), np.array(grid.bmax)
    pts = np.concatenate([g["pts"], rng.uniform(lo, hi, (400_000, 3))]).astype(np.float32)
    before = N.get_tuning()
    try:
        for n in (1, 255, 257, len(pts)):
            x = torch.tensor(pts[:n], device="cuda")
            out = {}
            for walk in (1, 2):
                N.set_tuning(query_walk=walk)
                c = grid.query_candidates(x, mode=4)
                q = grid.query_tensors(x, mode=4, unit=True, witness=True, valid=True)
                torch.cuda.synchronize()
                out[walk] = {k: v.cpu().numpy() for k, v in c.items()}
                out[walk].update({"q_" + k: v.cpu().numpy() for k, v in q.items()})
            for k in out[1]:
                assert np.array_equal(out[1][k], out[2][k], equal_nan=True), (n, k)
    finally:
        N.set_tuning(**before)
