"""The benchmarked query configurations at their own sizes, against the oracle.

* Hollow cylinder (34,816 triangles), dense 128x128x64, all 1,000,000
  Tricubic points of the benchmark (surface points offset along the face
  normal by N(0, (2h)^2), seed 1), queried exactly as the benchmark does:
  float32 points, gap + raw gradient + valid, through ``sdfo_query`` (the
  persistent walk kernel, the default for float32 points).
* Cube 0.1 m, dense 64^3 with 4 voxels of padding, 100,000 uniform points in
  the grid box (seed 0), Trilinear, same outputs.

Each is compared with two oracles on the same points:
* the reference's own ``SdfOracle::queryFast`` (SdfOracle.cpp:524-596,
  932-1092), compiled unmodified in oracle/_ref, on the reference's FP64
  grid: valid flags exactly, gap within 1e-5 * max(|gap|, h) (FP32 storage
  rounding included), and the unit normal (the reference returns only
  gradient / |gradient|) within 2e-5 * max(1, 1 / |gradient|);
* the C restatement (oracle/_port) in FP64 on the FP32 payload the GPU
  holds: valid exactly, gap within 1e-5 * max(|gap|, h), raw gradient within
  1e-5 * max(|gradient|, 1).
The restatement's normalised gradient is also checked against the
reference's unit normal at this size, which pins the restatement here.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_query(grid, pts, mode):
    import torch

    x = torch.tensor(pts, dtype=torch.float32, device="cuda")
    out = grid.query_tensors(x, mode=mode, unit=False, witness=False, valid=True)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def _compare(gpu, port_out, ref_out, h):
    valid = port_out["valid"]
    gap_ref, unit_ref, _, valid_ref = ref_out
    assert np.array_equal(valid, valid_ref), "oracle restatement valid flags vs reference"
    assert np.array_equal(gpu["valid"].astype(bool), valid_ref), "valid flags vs reference"
    v = valid_ref
    gap = gpu["gap"].astype(np.float64)
    grad = gpu["grad"].astype(np.float64)
    # against the restatement on the FP32 payload
    assert np.all(np.abs(gap - port_out["gap"]) <= 1e-5 * np.maximum(np.abs(port_out["gap"]), h))
    assert np.all(np.abs(grad - port_out["grad"]) <=
                  1e-5 * np.maximum(np.abs(port_out["grad"]), 1.0))
    # against the reference's FP64 grid (storage rounding included)
    assert np.all(np.abs(gap[v] - gap_ref[v]) <= 1e-5 * np.maximum(np.abs(gap_ref[v]), h))
    gn = np.linalg.norm(grad[v], axis=1, keepdims=True)
    unit = grad[v] / np.maximum(gn, 1e-30)
    tol = 2e-5 * np.maximum(1.0, 1.0 / np.maximum(gn, 1e-30))
    assert np.all(np.abs(unit - unit_ref[v]) <= tol)
    # the restatement's own normalised gradient reproduces the reference's
    pgn = np.linalg.norm(port_out["grad"][v], axis=1, keepdims=True)
    punit = port_out["grad"][v] / np.maximum(pgn, 1e-30)
    assert np.all(np.abs(punit - unit_ref[v]) <= 2e-5 * np.maximum(1.0, 1.0 / np.maximum(pgn, 1e-30)))
    # invalid points are zeroed by the kernel (prototype convention)
    assert np.all(gpu["gap"][~v] == 0.0) and np.all(gpu["grad"][~v] == 0.0)


def test_hollow_cylinder_1m_tricubic_vs_reference(cuda, port, ref):
    from sdfo import SdfGrid
    from sdfo import workloads as W

    c = W.c2_cylinder()
    grid = SdfGrid.build_dense(c["verts"], c["tris"], **c["dense"])
    assert grid.shape == (128, 128, 64)
    h = float(grid.voxel[0])
    pts = W.c2_points(c["verts"], c["tris"], h, 1_000_000, seed=1)
    assert pts.shape == (1_000_000, 3) and pts.dtype == np.float32
    gpu = _device_query(grid, pts, 3)

    R = ref.build_dense(c["verts"], c["tris"], **c["dense"])
    ref_out = R.query(3, pts.astype(np.float64))
    P = port.build_dense(c["verts"], c["tris"], **c["dense"])
    d = grid.export_dense()
    assert np.array_equal(d["phi"], P["phi"]) and np.array_equal(d["normal"], P["normal"])
    phi32 = P["phi"].astype(np.float32).astype(np.float64)
    n32 = P["normal"].astype(np.float32).astype(np.float64)
    port_out = port.query_dense(P["spec"], phi32, n32, None, 3, pts.astype(np.float64))
    _compare(gpu, port_out, ref_out, h)
    # the workload's points lie near the surface: almost all are valid
    assert ref_out[3].mean() > 0.99


def test_cube64_100k_trilinear_vs_reference(cuda, port, ref):
    from sdfo import SdfGrid
    from sdfo import workloads as W

    c = W.c1_cube64()
    grid = SdfGrid.build_dense(c["verts"], c["tris"], **c["build"])
    assert grid.shape == (64, 64, 64)
    h = float(grid.voxel[0])
    pts = W.c1_points(grid.bmin, grid.bmax, 100_000, seed=0)
    gpu = _device_query(grid, pts, 2)

    R = ref.build_dense(c["verts"], c["tris"], **c["build"])
    ref_out = R.query(2, pts.astype(np.float64))
    P = port.build_dense(c["verts"], c["tris"], **c["build"])
    phi32 = P["phi"].astype(np.float32).astype(np.float64)
    n32 = P["normal"].astype(np.float32).astype(np.float64)
    port_out = port.query_dense(P["spec"], phi32, n32, None, 2, pts.astype(np.float64))
    _compare(gpu, port_out, ref_out, h)
    # (63/64)^3 of the box has all eight corners inside the grid
    assert abs(ref_out[3].mean() - (63.0 / 64.0) ** 3) < 0.01
