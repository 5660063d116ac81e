"""GPU queries (all four modes, dense and sparse) against the oracle.

The oracle runs in FP64 on the same stored payload (the FP32 values the GPU
holds, widened), so the comparison isolates the kernels' FP32 arithmetic:
valid flags must match exactly; gap within 1e-5 * max(|gap|, h); gradient,
unit normal within 1e-5 * max(|.|, 1); interpolant Hessian within
2e-5 * (|H| + 1/h).  A second comparison against the FP64 grid states the
storage rounding on top, with the same bounds."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

MODES = [0, 1, 2, 3]


def _dense_fp32(g):
    phi = g["phi"].astype(np.float32).astype(np.float64)
    nrm = g["normal"].astype(np.float32).astype(np.float64)
    hes = g["hessian"].astype(np.float32).astype(np.float64)
    return phi, nrm, hes


def _check(gpu, ref, h, pts, modes_hess=True):
    valid = ref["valid"]
    assert np.array_equal(gpu["valid"].astype(bool), valid)
    gap = gpu["gap"].astype(np.float64)
    assert np.all(np.abs(gap - ref["gap"]) <= 1e-5 * np.maximum(np.abs(ref["gap"]), h))
    grad = gpu["grad"].astype(np.float64)
    assert np.all(np.abs(grad - ref["grad"]) <= 1e-5 * np.maximum(np.abs(ref["grad"]), 1.0))
    if "unit" in gpu:
        # grad/|grad| amplifies the gradient error by 1/|grad|: where the
        # gradient (nearly) vanishes (symmetry points) the direction is not
        # determined; the bound scales accordingly
        unit = gpu["unit"].astype(np.float64)
        gn = np.linalg.norm(ref["grad"], axis=1, keepdims=True)
        tol = 2e-5 * np.maximum(1.0, 1.0 / np.maximum(gn, 1e-30))
        assert np.all(np.abs(unit - ref["unit"]) <= tol)
        assert np.allclose(np.linalg.norm(unit[valid], axis=1), 1.0, atol=1e-6)
    if "witness" in gpu:
        # p - gap * unit: FP32 rounding of p plus |gap| times the unit bound
        w = gpu["witness"].astype(np.float64)
        scale = np.abs(pts).max() + h
        gn = np.linalg.norm(ref["grad"], axis=1, keepdims=True)
        utol = 2e-5 * np.maximum(1.0, 1.0 / np.maximum(gn, 1e-30))
        tol = 1e-6 * scale + 1e-5 * h + np.abs(ref["gap"])[:, None] * utol
        assert np.all(np.abs(w - ref["witness"]) <= tol)
    if "hess" in gpu and modes_hess:
        H = gpu["hess"].astype(np.float64)
        assert np.all(np.abs(H - ref["hess"]) <= 2e-5 * (np.abs(ref["hess"]) + 1.0 / h))


def _gpu_query(grid, pts, mode, f64=False):
    import torch

    t = torch.tensor(pts, dtype=torch.float64 if f64 else torch.float32, device="cuda")
    out = grid.query_tensors(t, mode=mode, unit=True, witness=True, valid=True, hess=True)
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("name", ["cube", "cyl", "torus"])
@pytest.mark.parametrize("mode", MODES)
def test_dense_query_vs_oracle(cuda, port, name, mode):
    from sdfo import SdfGrid

    g = golden(f"dense_{name}.npz")
    spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    grid = SdfGrid.from_dense(spec, g["phi"], g["normal"], g["hessian"], g["witness"])
    pts = g["pts"]  # FP32-representable, includes voxel centres and cell corners
    h = float(g["voxel"][0])
    phi, nrm, hes = _dense_fp32(g)
    ref32 = port.query_dense(spec, phi, nrm, hes, mode, pts)
    ref32["hess"] = ref32["hess"]
    gpu = _gpu_query(grid, pts, mode)
    gpu["hess"] = gpu["hess"].reshape(-1, 3, 3)
    _check(gpu, ref32, h, pts)
    # against the FP64 grid: storage rounding included
    ref64 = port.query_dense(spec, g["phi"], g["normal"], g["hessian"], mode, pts)
    _check({k: gpu[k] for k in ("valid", "gap", "grad", "unit")}, ref64, h, pts)
    # float64 points give the same cells and values
    gpu64 = _gpu_query(grid, pts, mode, f64=True)
    assert np.array_equal(gpu64["valid"], gpu["valid"])
    assert np.allclose(gpu64["gap"], gpu["gap"], rtol=0, atol=1e-6 * h)


@pytest.mark.parametrize("name", ["cube", "cyl"])
@pytest.mark.parametrize("mode", MODES)
def test_sparse_query_vs_oracle(cuda, port, name, mode):
    from sdfo import SdfGrid

    g = golden(f"sparse_{name}.npz")
    spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    bd = int(g["block_dim"])
    grid = SdfGrid.from_sparse(spec, bd, g["ijk"], g["phi"], g["normal"], g["hessian"],
                               int(g["halo"]), float(g["band"]))
    pts = g["pts"]
    h = float(g["voxel"][0])
    ref = port.query_sparse(spec, bd, g["ijk"], g["phi"], g["normal"], g["hessian"], mode, pts)
    gpu = _gpu_query(grid, pts, mode)
    gpu["hess"] = gpu["hess"].reshape(-1, 3, 3)
    _check(gpu, ref, h, pts)
    assert ref["valid"].any() and not ref["valid"].all()


@pytest.mark.parametrize("mode", MODES)
def test_queries_match_reference_golden(cuda, mode):
    """Straight against SdfOracle::queryFast results recorded from the reference."""
    from sdfo import SdfGrid

    g = golden("dense_torus.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    grid = SdfGrid.from_dense(spec, g["phi"], g["normal"], g["hessian"], g["witness"])
    gpu = _gpu_query(grid, g["pts"], mode)
    h = float(g["voxel"][0])
    v = g[f"q{mode}_valid"]
    assert np.array_equal(gpu["valid"].astype(bool), v)
    assert np.all(np.abs(gpu["gap"] - g[f"q{mode}_gap"]) <= 1e-5 * np.maximum(np.abs(g[f"q{mode}_gap"]), h))
    assert np.all(np.abs(gpu["unit"] - g[f"q{mode}_normal"]) <= 1e-5 * np.maximum(np.abs(g[f"q{mode}_normal"]), 1.0))


def test_query_batch_duck_type_matches_prototype(cuda):
    """SdfGrid.query_batch vs the prototype's TrilinearSDFGrid.query_batch."""
    from sdfo import SdfGrid

    g = golden("prototype_cube32.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    grid = SdfGrid.from_dense(spec, g["phi"], g["normal"])
    gq, raw, gn, unit, valid = grid.query_batch(g["pts"])
    h = float(g["voxel"][0])
    assert np.array_equal(valid, g["valid"])
    assert np.all(np.abs(gq - g["g"]) <= 1e-5 * np.maximum(np.abs(g["g"]), h))
    assert np.all(np.abs(raw - g["raw_grad"]) <= 1e-5 * np.maximum(np.abs(g["raw_grad"]), 1.0))
    assert np.all(np.abs(gn - g["grad_norm"]) <= 1e-5 * np.maximum(g["grad_norm"], 1.0))
    assert np.all(np.abs(unit - g["unit"]) <= 1e-5)
    assert np.all(unit[~valid] == np.array([0.0, 0.0, 1.0]))
    s = grid.query(g["pts"][0])
    assert len(s) == 5


def test_invalid_points_and_edges(cuda, port):
    from sdfo import SdfGrid

    g = golden("dense_cube.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    grid = SdfGrid.from_dense(spec, g["phi"], g["normal"], g["hessian"])
    pts = np.array([[np.nan, 0, 0], [np.inf, 0, 0], [-np.inf, 0, 0], [1e30, 0, 0], [0, 0, -1e30],
                    g["bmin"], g["bmax"], [0.0, 0.0, 0.0]], dtype=np.float32)
    for mode in MODES:
        r = _gpu_query(grid, pts, mode)
        assert not r["valid"][:6].any()
        assert np.all(r["gap"][:6] == 0) and np.all(r["grad"][:6] == 0)
        assert np.all(r["unit"][:6] == np.array([1, 0, 0], np.float32))
        assert r["valid"][7]
    # empty batch is a no-op
    import torch

    out = grid.query_tensors(torch.zeros((0, 3), device="cuda"), mode=3)
    assert out["gap"].numel() == 0


def test_host_path_matches_device_path(cuda):
    from sdfo import SdfGrid

    g = golden("dense_cyl.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    grid = SdfGrid.from_dense(spec, g["phi"], g["normal"], g["hessian"])
    pts = g["pts"].astype(np.float32)
    host = grid.query_host(pts, mode=3)
    dev = _gpu_query(grid, pts, 3)
    assert np.array_equal(host["gap"], dev["gap"])
    assert np.array_equal(host["grad"], dev["grad"])
    assert np.array_equal(host["valid"], dev["valid"].astype(bool))


def test_fp16_sparse_storage_error_bound(cuda, port):
    """FP16 brick payload: gap error stated against the FP64 oracle."""
    from sdfo import SdfGrid

    g = golden("sparse_cyl.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    bd = int(g["block_dim"])
    grid = SdfGrid.from_sparse(spec, bd, g["ijk"], g["phi"], g["normal"], g["hessian"])
    g16 = grid.to_fp16()
    pts = g["pts"]
    h = float(g["voxel"][0])
    ref = port.query_sparse(port.GridSpec(**spec), bd, g["ijk"], g["phi"], g["normal"],
                            g["hessian"], 3, pts)
    r16 = _gpu_query(g16, pts, 3)
    v = ref["valid"]
    assert np.array_equal(r16["valid"].astype(bool), v)
    # per-brick affine phi in FP16: |d phi| <= 2^-11 * half-range of the brick's
    # phi (<= sqrt(3) * bd * h), normals to 2^-11
    bound = 2.0 ** -11 * np.sqrt(3.0) * bd * h * 1.5
    assert np.max(np.abs(r16["gap"][v] - ref["gap"][v])) <= bound
    d = g16.export_sparse()
    assert np.max(np.abs(d["phi"] - g["phi"])) <= bound


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("mode", [2, 3])
@pytest.mark.parametrize("n", [255, 256 * 41, 256 * 41 + 97])
def test_pipelined_dense_query_is_bit_identical(cuda, mode, n, walk):
    """Float32 points on a dense grid take the persistent walk kernel (the
    default) or, with the walk off, the persistent bulk-copy pipeline for
    whole tiles of 256 (the rest in one extra CTA); the Hessian-writing
    forward always takes the pipeline.  The same points as float64 (the plain
    kernel throughout) give bit-identical gap, gradient, valid flags and
    linearisation Hessians."""
    import torch

    from sdfo import SdfGrid
    from sdfo import _native as N
    from sdfo import meshes as M

    v, t = M.torus(0.05, 0.01, 48, 12)
    grid = SdfGrid.build_dense(v, t, target_resolution=40, max_resolution=40)
    rng = np.random.default_rng(n)
    p32 = torch.tensor(rng.uniform(grid.bmin, grid.bmax, (n, 3)).astype(np.float32), device="cuda")
    before = N.get_tuning()
    try:
        N.set_tuning(query_walk=walk)
        a = grid.query_tensors(p32, mode=mode)
        lin = grid.query_linearize(p32, mode=mode)
        torch.cuda.synchronize()
    finally:
        N.set_tuning(**before)
    b = grid.query_tensors(p32.double(), mode=mode)
    for k in ("gap", "grad", "valid"):
        assert torch.equal(a[k], b[k]), k
    h = grid.query_tensors(p32.double(), mode=mode, hess=True)
    assert torch.equal(lin["gap"], h["gap"]) and torch.equal(lin["grad"], h["grad"])
    H = h["hess"].reshape(n, 9)[:, [0, 1, 2, 4, 5, 8]]
    assert torch.equal(lin["hess6"], H)


@pytest.mark.parametrize("mode", [2, 3])
def test_sparse_pair_records_bit_identical(cuda, mode):
    """Sparse grids with the x-pair records (one 256-bit load per Tricubic
    row) and without them (a tuning knob) answer every query bit for bit
    alike, including cells on brick faces and next to missing bricks."""
    import torch

    from sdfo import SdfGrid
    from sdfo import _native as N

    g = golden("sparse_cyl.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    before = N.get_tuning()
    out = {}
    rng = np.random.default_rng(5)
    pts = np.concatenate([g["pts"], rng.uniform(g["bmin"], g["bmax"], (60_000, 3))]).astype(np.float32)
    x = torch.tensor(pts, device="cuda")
    try:
        for pairs in (1, 2):
            N.set_tuning(sparse_pair_records=pairs)
            grid = SdfGrid.from_sparse(spec, int(g["block_dim"]), g["ijk"], g["phi"], g["normal"],
                                       g["hessian"])
            o = grid.query_tensors(x, mode=mode, unit=True, witness=True, valid=True, hess=True)
            torch.cuda.synchronize()
            out[pairs] = {k: v.cpu().numpy() for k, v in o.items()}
    finally:
        N.set_tuning(**before)
    assert out[1]["valid"].sum() > 1000
    for k in out[1]:
        assert np.array_equal(out[1][k], out[2][k], equal_nan=True), k


@pytest.mark.parametrize("mode", [2, 3])
def test_query_walk_bit_identical(cuda, mode):
    """The persistent walk kernel for FP32-point queries (the default; a
    tuning knob) answers every query bit for bit as the per-tile kernels do
    (staged on sparse grids, the bulk-copy pipeline on dense ones): sparse
    FP32 and FP16 pools and a dense grid, every output (the full and the
    symmetric Hessian included), and batch sizes below one tile, between
    tiles and above the resident CTA count."""
    import torch

    from sdfo import SdfGrid
    from sdfo import _native as N
    from sdfo import workloads as W

    g = golden("sparse_cyl.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    grid = SdfGrid.from_sparse(spec, int(g["block_dim"]), g["ijk"], g["phi"], g["normal"], g["hessian"])
    c = W.c2_cylinder()
    dense = SdfGrid.build_dense(c["verts"], c["tris"], mode=3, target_resolution=64, max_resolution=64)
    grids = [grid, grid.to_fp16(), dense]
    rng = np.random.default_rng(8)
    before = N.get_tuning()
    try:
        for gr in grids:
            lo, hi = np.array(gr.bmin), np.array(gr.bmax)
            pts = np.concatenate([g["pts"], rng.uniform(lo, hi, (700_000, 3))]).astype(np.float32)
            for n in (1, 255, 257, 40_000, len(pts)):
                x = torch.tensor(pts[:n], device="cuda")
                out = {}
                for walk in (1, 2):
                    N.set_tuning(query_walk=walk)
                    o = gr.query_tensors(x, mode=mode, unit=True, witness=True, valid=True)
                    fast = gr.query_tensors(x, mode=mode, valid=True)
                    h = gr.query_tensors(x, mode=mode, valid=True, hess=True)
                    lin = gr.query_linearize(x, mode=mode)
                    torch.cuda.synchronize()
                    out[walk] = {k: v.cpu().numpy() for k, v in o.items()}
                    out[walk].update({"f_" + k: v.cpu().numpy() for k, v in fast.items()})
                    out[walk].update({"h_" + k: v.cpu().numpy() for k, v in h.items()})
                    out[walk].update({"lin_" + k: v.cpu().numpy() for k, v in lin.items()})
                if n == len(pts):
                    assert out[1]["valid"].sum() > 1000
                for k in out[1]:
                    assert np.array_equal(out[1][k], out[2][k], equal_nan=True), (gr.storage, gr.is_sparse, n, k)
    finally:
        N.set_tuning(**before)
