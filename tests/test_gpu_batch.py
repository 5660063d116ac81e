"""Batched sparse build (sdfo_grid_build_sparse_batched) over gear prisms of
uneven size and resolution: every grid of the batch must equal the
single-mesh build of its mesh bit for bit (occupancy, table, payload,
Hessian), in both BVH modes, and the single-mesh build is pinned to the
oracle (test_gpu_build); a few batch members are also compared with the
oracle directly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _set_mode(m):
    from sdfo import _native as N

    N.check(N.load().sdfo_set_bvh_mode(m))


def _mesh_args(g):
    return dict(verts=g["verts"], tris=g["tris"], **g["sparse"])


def _equal(a, b):
    da, db = a.export_sparse(), b.export_sparse()
    assert a.shape == b.shape and a.block_count == b.block_count
    assert np.array_equal(np.array(a.bmin), np.array(b.bmin))
    for k in ("ijk", "phi", "normal", "hessian"):
        assert np.array_equal(da[k], db[k]), k


@pytest.mark.parametrize("bvh", [0, 1])
def test_batch_equals_single_builds(cuda, bvh):
    from sdfo import SdfGrid
    from sdfo import workloads as W

    gears = W.c4_gears(n_gears=12, seed=3)
    _set_mode(bvh)
    try:
        grids = SdfGrid.build_sparse_batched([_mesh_args(g) for g in gears], mode=3)
        assert len(grids) == len(gears)
        for g, grid in zip(gears, grids):
            single = SdfGrid.build_sparse(g["verts"], g["tris"], mode=3, **g["sparse"])
            _equal(grid, single)
            s = grid.build_stats()
            assert s["triangles"] == len(g["tris"])
    finally:
        _set_mode(0)


def test_batch_members_vs_oracle(cuda, port):
    from sdfo import SdfGrid
    from sdfo import workloads as W

    gears = W.c4_gears(n_gears=5, seed=3)
    _set_mode(0)
    grids = SdfGrid.build_sparse_batched([_mesh_args(g) for g in gears])
    for g, grid in list(zip(gears, grids))[:3]:
        P = port.build_sparse(g["verts"], g["tris"], **g["sparse"])
        d = grid.export_sparse()
        assert np.array_equal(d["ijk"], P["ijk"])
        assert np.array_equal(d["phi"], P["phi"])
        assert np.array_equal(d["normal"], P["normal"])
        assert np.array_equal(d["hessian"], P["hessian"])


def test_batch_handles_outlive_each_other(cuda):
    """The grids share one arena: closing some keeps the others valid."""
    import torch

    from sdfo import SdfGrid
    from sdfo import meshes as M

    ms = [M.cube(0.1), M.torus(0.05, 0.01, 48, 12), M.gear_prism(24, 0.05, 0.01, 3000)]
    args = [dict(verts=v, tris=t, target_resolution=32, max_resolution=32, band_voxels=3)
            for v, t in ms]
    grids = SdfGrid.build_sparse_batched(args, mode=3)
    ref = [g.export_sparse()["phi"].copy() for g in grids]
    grids[0].close()
    grids[1].close()
    x = torch.zeros((4, 3), device="cuda")
    out = grids[2].query_tensors(x, mode=3)
    torch.cuda.synchronize()
    assert np.array_equal(grids[2].export_sparse()["phi"], ref[2])
    assert out["gap"].shape == (4,)


def test_batch_rejects_mixed_block_dims(cuda):
    from sdfo import SdfGrid
    from sdfo import _native as N
    from sdfo import meshes as M

    v, t = M.cube(0.1)
    with pytest.raises(N.SdfoError, match="same blockDim"):
        SdfGrid.build_sparse_batched([dict(verts=v, tris=t, target_resolution=32, block_dim=8),
                                      dict(verts=v, tris=t, target_resolution=32, block_dim=4)])


def test_c4_full_batch(cuda):
    """All 256 gears (4.4M triangles, 64^3..256^3) in one batched build; 16
    of them compared with their single-mesh builds."""
    from sdfo import SdfGrid
    from sdfo import workloads as W

    gears = W.c4_gears()
    _set_mode(0)
    grids = SdfGrid.build_sparse_batched([_mesh_args(g) for g in gears], mode=3)
    assert len(grids) == 256
    assert all(g.block_count > 0 for g in grids)
    for i in range(0, 256, 16):
        single = SdfGrid.build_sparse(gears[i]["verts"], gears[i]["tris"], mode=3,
                                      **gears[i]["sparse"])
        _equal(grids[i], single)


def _rotation(rng):
    """Rodrigues rotation about a random axis by a random angle."""
    k = rng.normal(size=3)
    k /= np.linalg.norm(k)
    a = rng.uniform(0.0, np.pi)
    K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
    return np.eye(3) + np.sin(a) * K + (1.0 - np.cos(a)) * (K @ K)


def _batch_case(port, n_points=4096, seed=9):
    """Five gears (sparse FP32, one of them re-encoded FP16) and a dense cube,
    each with near-surface points in its own frame and a random pose."""
    from sdfo import SdfGrid
    from sdfo import meshes as M
    from sdfo import workloads as W

    gears = W.c4_gears(n_gears=5, seed=3)
    _set_mode(0)
    grids = SdfGrid.build_sparse_batched([_mesh_args(g) for g in gears], mode=3)
    grids[2] = grids[2].to_fp16()
    cv, ct = M.cube(0.1)
    grids.append(SdfGrid.build_dense(cv, ct, target_resolution=48, max_resolution=48, mode=3))
    meshes = [(g["verts"], g["tris"]) for g in gears] + [(cv, ct)]
    rng = np.random.default_rng(seed)
    local, world, R, t = [], [], [], []
    for (v, tr), grid in zip(meshes, grids):
        p = W.near_surface_points(v, tr, float(grid.voxel[0]), n_points, int(rng.integers(1 << 30)))
        Rg = _rotation(rng)
        tg = rng.uniform(-0.2, 0.2, 3)
        x = (p.astype(np.float64) @ Rg.T + tg).astype(np.float32)
        world.append(x)
        R.append(Rg)
        t.append(tg)
        local.append((x.astype(np.float64) - tg) @ Rg)  # R^T (x - t), row vectors
    return grids, local, world, np.array(R), np.array(t)


def _oracle_local(port, grid, pts):
    spec = port.GridSpec(bmin=np.array(grid.bmin), bmax=np.array(grid.bmax),
                         voxel=np.array(grid.voxel), shape=tuple(grid.shape))
    if grid.is_sparse:
        d = grid.export_sparse()
        return port.query_sparse(spec, grid.block_dim, d["ijk"], d["phi"].astype(np.float64),
                                 d["normal"].astype(np.float64), None, 3, pts)
    d = grid.export_dense()
    return port.query_dense(spec, d["phi"].astype(np.float32).astype(np.float64),
                            d["normal"].astype(np.float32).astype(np.float64), None, 3, pts)


def test_query_batch_with_poses_vs_oracle(cuda, port):
    import torch

    from sdfo.batch import QueryBatch, pack_poses

    grids, local, world, R, t = _batch_case(port)
    counts = [len(w) for w in world]
    qb = QueryBatch(grids, counts)
    x = torch.tensor(np.concatenate(world), device="cuda")
    gap, grad, valid = qb.run(x, pack_poses(R, t))
    gap, grad, valid = gap.cpu().numpy(), grad.cpu().numpy(), valid.cpu().numpy().astype(bool)
    off = np.concatenate([[0], np.cumsum(counts)])
    for g, grid in enumerate(grids):
        s = slice(off[g], off[g + 1])
        ref = _oracle_local(port, grid, local[g])
        v = ref["valid"]
        assert v.mean() > 0.9
        assert np.array_equal(valid[s], v)
        h = float(grid.voxel[0])
        fp16 = grid.storage == 1
        gtol = (2.0 ** -11 * 8 * h if fp16 else 0.0) + 1e-5 * np.maximum(np.abs(ref["gap"]), h)
        assert np.all(np.abs(gap[s] - ref["gap"])[v] <= gtol[v])
        gw = ref["grad"] @ R[g].T
        ntol = (0.02 if fp16 else 1e-5) * np.maximum(np.abs(gw), 1.0)
        assert np.all(np.abs(grad[s] - gw)[v] <= ntol[v])
        assert np.all(gap[s][~v] == 0)


def test_query_batch_identity_pose_equals_single_queries(cuda, port):
    import torch

    from sdfo.batch import QueryBatch

    grids, local, _, _, _ = _batch_case(port, n_points=1000)
    qb = QueryBatch(grids, [len(p) for p in local])
    pts32 = [p.astype(np.float32) for p in local]
    gap, grad, valid = qb.run(torch.tensor(np.concatenate(pts32), device="cuda"))
    off = np.concatenate([[0], np.cumsum([len(p) for p in pts32])])
    for g, grid in enumerate(grids):
        one = grid.query_tensors(torch.tensor(pts32[g], device="cuda"), mode=3, valid=True)
        s = slice(off[g], off[g + 1])
        assert torch.equal(valid[s], one["valid"])
        assert torch.allclose(gap[s], one["gap"], rtol=0, atol=1e-6 * float(grid.voxel[0]))
        assert torch.allclose(grad[s], one["grad"], rtol=0, atol=1e-6)


@pytest.mark.parametrize("kind", ["sparse", "sparse16", "dense"])
def test_query_batch_ragged_counts(cuda, kind):
    """The persistent batch kernel walks runs of tiles in grid-stride order:
    grids with no queries between others, tails shorter than a CTA, more
    tiles than resident CTAs (several grid changes per CTA) and repeated
    grids must all answer as the single-grid query does, for every launch
    shape and run length, and for batches of one layout (the kernel is
    specialised on it)."""
    import torch

    from sdfo import SdfGrid
    from sdfo import meshes as M
    from sdfo import workloads as W
    from sdfo.batch import QueryBatch

    if kind in ("sparse", "sparse16"):
        gears = W.c4_gears(n_gears=3, seed=5)
        _set_mode(0)
        base = SdfGrid.build_sparse_batched([_mesh_args(g) for g in gears], mode=3)
        if kind == "sparse16":
            base = [b.to_fp16() for b in base]
        meshes = [(g["verts"], g["tris"]) for g in gears]
    else:
        cv, ct = M.cube(0.1)
        base = [SdfGrid.build_dense(cv, ct, target_resolution=40, max_resolution=40, mode=3)]
        meshes = [(cv, ct)]
    counts = [0, 1, 0, 257, 0, 300_000, 3, 128, 129, 0, 100_000, 0]
    which = [i % len(base) for i in range(len(counts))]
    rng = np.random.default_rng(21)
    pts = []
    for c, w in zip(counts, which):
        v, tr = meshes[w]
        p = W.near_surface_points(v, tr, float(base[w].voxel[0]), max(c, 1), int(rng.integers(1 << 30)))
        pts.append(p[:c].astype(np.float32))
    qb = QueryBatch([base[w] for w in which], counts)
    for bad in (0, 3, 128):
        with pytest.raises(RuntimeError, match="run length"):
            qb.set_run(bad)
    x = torch.tensor(np.concatenate(pts), device="cuda")
    off = np.concatenate([[0], np.cumsum(counts)])
    single = []
    for g, w in enumerate(which):
        if counts[g]:
            single.append(base[w].query_tensors(torch.tensor(pts[g], device="cuda"), mode=3, valid=True))
        else:
            single.append(None)
    for threads, run in ((128, 1), (256, 1), (512, 1), (128, 4), (256, 64)):
        qb.set_threads(threads)
        qb.set_run(run)
        gap, grad, valid = qb.run(x)
        for g, w in enumerate(which):
            if not counts[g]:
                continue
            one, s = single[g], slice(off[g], off[g + 1])
            h = float(base[w].voxel[0])
            assert torch.equal(valid[s], one["valid"]), (threads, run, g)
            assert torch.allclose(gap[s], one["gap"], rtol=0, atol=1e-6 * h), (threads, run, g)
            assert torch.allclose(grad[s], one["grad"], rtol=0, atol=1e-6), (threads, run, g)


def test_query_batch_cuda_graph_and_threads(cuda, port):
    import torch

    from sdfo.batch import QueryBatch, pack_poses
    from sdfo.tune import tune_query_batch

    grids, _, world, R, t = _batch_case(port, n_points=2000)
    qb = QueryBatch(grids, [len(w) for w in world])
    x = torch.tensor(np.concatenate(world), device="cuda")
    poses = pack_poses(R, t)
    eager = qb.run(x, poses)
    graph, out = qb.capture(x, poses)
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager, out):
        assert torch.equal(a, b)
    # new inputs in place, replay again
    x.add_(1e-4)
    eager2 = qb.run(x, poses)
    graph.replay()
    torch.cuda.synchronize()
    for a, b in zip(eager2, out):
        assert torch.equal(a, b)
    # every launch shape gives the same answer; the tuner keeps one of them
    for threads in (128, 256, 512):
        qb.set_threads(threads)
        for run in (1, 2, 8, 64):
            qb.set_run(run)
            for a, b in zip(eager2, qb.run(x, poses)):
                assert torch.equal(a, b)
    res = tune_query_batch(qb, x, poses, reps=3, warmup=1)
    assert res["threads"] in (128, 256, 512) and qb.threads == res["threads"]
    assert res["run"] in (1, 2, 4, 8) and qb.run_tiles == res["run"]


def test_tuners_run(cuda):
    import torch

    from sdfo import meshes as M
    from sdfo import workloads as W
    from sdfo.tune import tune_block_dim, tune_fill_ctas

    v, t = M.torus(0.05, 0.01, 48, 12)
    pts = torch.tensor(W.near_surface_points(v, t, 0.12 / 64, 20000, 1), device="cuda")
    r = tune_block_dim(v, t, pts, reps=2, warmup=1, target_resolution=64, max_resolution=64,
                       band_voxels=3)
    assert r["block_dim"] in (4, 8, 16)
    gears = W.c4_gears(n_gears=6, seed=3)
    f = tune_fill_ctas([_mesh_args(g) for g in gears], candidates=(1, 2))
    assert f["ctas_per_sm"] in (1, 2)
    from sdfo import _native as N

    N.check(N.load().sdfo_set_fill_ctas_per_sm(0))
