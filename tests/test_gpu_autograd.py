"""Backward kernels behind torch.autograd (sdfo.autograd.sdf_query).

d/d(points): dL/dp = dgap * grad + H dgrad, checked against the FP64
oracle's analytic gradient and Hessian on the same payload (tolerance
1e-5 * max(|.|, 1) on the gradient part, 2e-5 * (|H| + 1/h) on the Hessian
part).  d/d(payload): the interpolants are linear in the stored {phi, n}, so
central differences of the loss w.r.t. single payload entries are exact up to
rounding; checked to 1e-3 relative."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _grid_and_ref(port, layout):
    from sdfo import SdfGrid

    if layout == "dense":
        g = golden("dense_torus.npz")
        spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
        grid = SdfGrid.from_dense(spec, g["phi"], g["normal"], g["hessian"])
        phi = g["phi"].astype(np.float32).astype(np.float64)
        nrm = g["normal"].astype(np.float32).astype(np.float64)

        def ref(mode, pts):
            return port.query_dense(spec, phi, nrm, None, mode, pts)
    else:
        g = golden("sparse_cyl.npz")
        spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
        bd = int(g["block_dim"])
        grid = SdfGrid.from_sparse(spec, bd, g["ijk"], g["phi"], g["normal"], g["hessian"])

        def ref(mode, pts):
            return port.query_sparse(spec, bd, g["ijk"], g["phi"], g["normal"], None, mode, pts)
    return grid, ref, g


@pytest.mark.parametrize("layout", ["dense", "sparse"])
@pytest.mark.parametrize("mode", [2, 3])
def test_point_gradient_vs_oracle(cuda, port, layout, mode):
    import torch

    from sdfo.autograd import sdf_query

    grid, ref, g = _grid_and_ref(port, layout)
    pts = g["pts"].astype(np.float32)
    rng = np.random.default_rng(5)
    wg = rng.normal(size=len(pts))
    wn = rng.normal(size=(len(pts), 3))
    x = torch.tensor(pts, device="cuda", requires_grad=True)
    gap, grad = sdf_query(grid, x, mode=mode)
    loss = (gap * torch.tensor(wg, device="cuda", dtype=torch.float32)).sum() + (
        grad * torch.tensor(wn, device="cuda", dtype=torch.float32)).sum()
    loss.backward()
    dp = x.grad.cpu().numpy().astype(np.float64)
    r = ref(mode, pts.astype(np.float64))
    h = float(g["voxel"][0])
    expect = wg[:, None] * r["grad"] + np.einsum("nab,nb->na", r["hess"], wn)
    tol = 1e-5 * np.abs(wg)[:, None] * np.maximum(np.abs(r["grad"]), 1.0) + \
        2e-5 * np.einsum("nab,nb->na", np.abs(r["hess"]) + 1.0 / h, np.abs(wn))
    v = r["valid"]
    assert np.all(np.abs(dp[v] - expect[v]) <= tol[v])
    assert np.all(dp[~v] == 0)


@pytest.mark.parametrize("layout", ["dense", "sparse"])
@pytest.mark.parametrize("mode", [2, 3])
def test_payload_gradient_vs_central_differences(cuda, port, layout, mode):
    import torch

    from sdfo.autograd import sdf_query

    grid, _, g = _grid_and_ref(port, layout)
    pts = g["pts"][:600].astype(np.float32)
    x = torch.tensor(pts, device="cuda")
    payload = grid.payload().clone().requires_grad_(True)
    gap, grad = sdf_query(grid, x, payload=payload, mode=mode)
    loss = gap.sum() + 0.5 * grad[:, 0].sum() - 0.25 * grad[:, 2].sum()
    loss.backward()
    G = payload.grad.cpu().numpy()
    touched = np.argwhere(np.abs(G).sum(1) > 0)[:, 0]
    assert len(touched) > 50
    rng = np.random.default_rng(3)
    eps = 1e-2
    with torch.no_grad():
        for vox in rng.choice(touched, 12, replace=False):
            for ch in ([0] if mode == 2 else [0, 1, 3]):
                base = payload.detach().clone()
                p1, p2 = base.clone(), base.clone()
                p1[vox, ch] += eps
                p2[vox, ch] -= eps
                l1 = _loss(grid, x, p1, mode)
                l2 = _loss(grid, x, p2, mode)
                fd = (l1 - l2) / (2 * eps)
                assert abs(fd - G[vox, ch]) <= 1e-3 * max(abs(G[vox, ch]), 1.0), (vox, ch, fd, G[vox, ch])


def _loss(grid, x, payload, mode):
    from sdfo.autograd import sdf_query

    gap, grad = sdf_query(grid, x, payload=payload.contiguous(), mode=mode)
    return float((gap.double().sum() + 0.5 * grad[:, 0].double().sum() - 0.25 * grad[:, 2].double().sum()).item())


@pytest.mark.parametrize("storage", ["dense", "sparse", "sparse_fp16"])
@pytest.mark.parametrize("mode", [2, 3])
def test_saved_and_regathered_backward_agree(cuda, port, storage, mode):
    """sdfo_query_backward_saved (elementwise from the forward's saved grad
    and Hessian, weights-only grid scatter) against sdfo_query_backward (the
    stencil gathered again): the same interpolant, so agreement to rounding."""
    import torch

    grid, _, g = _grid_and_ref(port, "dense" if storage == "dense" else "sparse")
    if storage == "sparse_fp16":
        grid = grid.to_fp16()
    pts = torch.tensor(g["pts"].astype(np.float32), device="cuda")
    n = pts.shape[0]
    gen = torch.Generator(device="cuda").manual_seed(11)
    dgap = torch.randn(n, device="cuda", generator=gen)
    dgrad = torch.randn((n, 3), device="cuda", generator=gen)
    saved = grid.query_linearize(pts, mode=mode)
    plain = grid.query_tensors(pts, mode=mode, valid=True)
    assert torch.equal(saved["valid"], plain["valid"])
    h = float(g["voxel"][0])
    assert float((saved["gap"] - plain["gap"]).abs().max()) <= 1e-6 * h
    assert float((saved["grad"] - plain["grad"]).abs().max()) <= 1e-6
    G1 = torch.zeros((grid.stored_voxels, 4), device="cuda")
    G2 = torch.zeros_like(G1)
    d1 = grid.query_backward_saved(pts, saved, dgap, dgrad, mode=mode, dgrid=G1)
    d2 = grid.query_backward(pts, dgap, dgrad, mode=mode, dgrid=G2)
    scale = float(d2.abs().max())
    assert float((d1 - d2).abs().max()) <= 1e-6 * scale
    assert float((G1 - G2).abs().max()) <= 1e-5 * max(float(G2.abs().max()), 1.0)
    v = saved["valid"].bool()
    assert torch.all(d1[~v] == 0)
    # each output alone
    d3 = grid.query_backward_saved(pts, saved, dgap, None, mode=mode)
    assert torch.allclose(d3, dgap[:, None] * saved["grad"], rtol=0, atol=1e-6 * scale)
    G3 = torch.zeros_like(G1)
    assert grid.query_backward_saved(pts, {"valid": saved["valid"]}, dgap, dgrad, mode=mode,
                                     dgrid=G3, want_points=False) is None
    assert float((G3 - G1).abs().max()) <= 1e-5 * max(float(G1.abs().max()), 1.0)


@pytest.mark.parametrize("n", [77, 256 * 301, 256 * 301 + 77])
def test_bulk_copy_backward_matches_regathered(cuda, port, n):
    """dL/dp from the saved linearisation alone (the bulk-copy pipeline for
    whole tiles of 256 queries, the staged kernel for the rest) against the
    regathering backward, with both upstream gradients, with dgap only and
    with dgrad only; the kernels' status word stays clear."""
    import ctypes

    import torch

    from sdfo import _native as N

    grid, _, g = _grid_and_ref(port, "sparse")
    rng = np.random.default_rng(n)
    base = g["pts"].astype(np.float32)
    pts = torch.tensor(base[rng.integers(0, len(base), n)], device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(n)
    dgap = torch.randn(n, device="cuda", generator=gen)
    dgrad = torch.randn((n, 3), device="cuda", generator=gen)
    saved = grid.query_linearize(pts, mode=3)
    for dg, dr in ((dgap, dgrad), (dgap, None), (None, dgrad)):
        d1 = grid.query_backward_saved(pts, saved, dg, dr, mode=3)
        d2 = grid.query_backward(pts, dg, dr, mode=3)
        scale = max(float(d2.abs().max()), 1e-9)
        assert float((d1 - d2).abs().max()) <= 1e-6 * scale
    torch.cuda.synchronize()
    flags = ctypes.c_uint32(7)
    N.check(N.load().sdfo_device_status(ctypes.byref(flags), 1))
    assert flags.value == 0


def test_regathering_backward_walk_bit_identical(cuda):
    """The persistent walk kernel of the regathering backward for dL/dp (the
    default; sdfo_tuning.query_walk) gives dL/dp bit for bit as the
    one-CTA-per-tile kernel does: dense and sparse FP32 / FP16 grids, each
    combination of upstream gradients, batch sizes below one tile, between
    tiles and above the resident CTA count."""
    import torch

    from conftest import golden
    from sdfo import SdfGrid
    from sdfo import _native as N
    from sdfo import workloads as W

    g = golden("sparse_cyl.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    sparse = SdfGrid.from_sparse(spec, int(g["block_dim"]), g["ijk"], g["phi"], g["normal"], g["hessian"])
    c = W.c2_cylinder()
    dense = SdfGrid.build_dense(c["verts"], c["tris"], mode=3, target_resolution=64, max_resolution=64)
    rng = np.random.default_rng(17)
    before = N.get_tuning()
    try:
        for gr in (sparse, sparse.to_fp16(), dense):
            lo, hi = np.array(gr.bmin), np.array(gr.bmax)
            pts = np.concatenate([g["pts"], rng.uniform(lo, hi, (600_000, 3))]).astype(np.float32)
            for n in (1, 255, 257, len(pts)):
                x = torch.tensor(pts[:n], device="cuda")
                gen = torch.Generator(device="cuda").manual_seed(n)
                dgap = torch.randn(n, device="cuda", generator=gen)
                dgrad = torch.randn((n, 3), device="cuda", generator=gen)
                for dg, dr in ((dgap, dgrad), (dgap, None), (None, dgrad)):
                    out = {}
                    for walk in (1, 2):
                        N.set_tuning(query_walk=walk)
                        out[walk] = gr.query_backward(x, dg, dr, mode=3).cpu().numpy()
                    assert np.array_equal(out[1], out[2]), (gr.storage, gr.is_sparse, n)
    finally:
        N.set_tuning(**before)
