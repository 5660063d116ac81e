"""sdfo_query_host_static: the host-buffer query that allocates no device
memory, for callers that cannot let a library call cudaMalloc (hosts that own
all GPU memory through their own pool, or forbid allocations inside their
step loop).  Its staging lives in a fixed device array inside the library.

Checked through the C ABI against sdfo_query_host (the allocating path) on
the same grid and points, with the query tolerances used elsewhere, on two
calls in a row (the array keeps the previous call's contents), with float32
and float64 points, on dense, sparse and contact-aware grids, and for the
size limit.  A fresh handle answered only through the static path leaves the
device's free memory and the library's block cache unchanged.  This file is
collected last so a run that stops at the first failure has already run
every other test."""
import ctypes

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _grid():
    from sdfo import SdfGrid

    g = golden("dense_torus.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    return SdfGrid.from_dense(spec, g["phi"], g["normal"], g["hessian"]), g


def _sparse_grid():
    from sdfo import SdfGrid

    g = golden("sparse_cube.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    grid = SdfGrid.from_sparse(spec, int(g["block_dim"]), g["ijk"], g["phi"], g["normal"],
                               g["hessian"])
    return grid, g


def _contact_aware_grid():
    import ast

    from sdfo import SdfGrid

    g = golden("ca_dense_cube.npz")
    grid = SdfGrid.build_contact_aware(g["verts"], g["tris"], g["corner_normals"], padding=0.1,
                                       **ast.literal_eval(str(g["params"])))
    return grid, g


def _held(lib):
    from sdfo import _native as N

    held = ctypes.c_int64(0)
    N.check(lib.sdfo_device_cache(-1, ctypes.byref(held)))
    return int(held.value)


def _static(lib, grid, pts, mode, with_grad=True, with_valid=True):
    from sdfo import _native as N

    n = len(pts)
    gap = np.full(n, np.nan, np.float32)
    grad = np.full((n, 3), np.nan, np.float32) if with_grad else None
    valid = np.full(n, 7, np.uint8) if with_valid else None
    p = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    N.check(lib.sdfo_query_host_static(grid.handle, mode, p(pts),
                                       1 if pts.dtype == np.float64 else 0, n, p(gap), p(grad),
                                       p(valid), None))
    return gap, grad, valid


def _close(a, b, h):
    gap, grad, valid = a
    assert np.array_equal(valid.astype(bool), b["valid"])
    assert np.all(np.abs(gap - b["gap"]) <= 1e-5 * np.maximum(np.abs(b["gap"]), h))
    assert np.all(np.abs(grad - b["grad"]) <= 1e-5 * np.maximum(np.abs(b["grad"]), 1.0))


@pytest.mark.parametrize("mode", [2, 3])
def test_static_staging_matches_allocating_path(cuda, mode):
    from sdfo import _native as N

    lib = N.load()
    grid, g = _grid()
    h = float(g["voxel"][0])
    rng = np.random.default_rng(17)
    pts1 = rng.uniform(g["bmin"], g["bmax"], (50_000, 3)).astype(np.float32)
    pts2 = rng.uniform(g["bmin"], g["bmax"], (20_000, 3)).astype(np.float32)
    ref1 = grid.query_host(pts1, mode=mode)
    ref2 = grid.query_host(pts2, mode=mode)
    # two calls in a row, the second smaller than the first
    _close(_static(lib, grid, pts1, mode), ref1, h)
    _close(_static(lib, grid, pts2, mode), ref2, h)
    _close(_static(lib, grid, pts1, mode), ref1, h)
    # float64 points and optional outputs
    pts64 = pts2.astype(np.float64)
    ref64 = grid.query_host(pts64, mode=mode)
    gap, grad, valid = _static(lib, grid, pts64, mode, with_grad=False, with_valid=False)
    assert grad is None and valid is None
    assert np.all(np.abs(gap - ref64["gap"]) <= 1e-5 * np.maximum(np.abs(ref64["gap"]), h))


def test_static_staging_limit(cuda):
    from sdfo import _native as N

    lib = N.load()
    grid, g = _grid()
    n = (32 << 20) // 12 + 1  # the float32 points alone exceed the 32 MiB array
    pts = np.zeros((n, 3), np.float32)
    gap = np.zeros(n, np.float32)
    rc = lib.sdfo_query_host_static(grid.handle, 3, ctypes.c_void_p(pts.ctypes.data), 0, n,
                                    ctypes.c_void_p(gap.ctypes.data), None, None, None)
    assert rc == -1
    assert "static limit" in N.last_error()
    # the entry point stays usable after a rejected call
    small = np.asarray(g["pts"][:100], np.float32)
    ref = grid.query_host(small, mode=3)
    _close(_static(lib, grid, small, 3), ref, float(g["voxel"][0]))


@pytest.mark.parametrize("kind,modes", [("sparse", (2, 3)), ("contact_aware", (4, 3))])
def test_static_staging_sparse_and_contact_aware(cuda, kind, modes):
    from sdfo import _native as N

    lib = N.load()
    grid, g = _sparse_grid() if kind == "sparse" else _contact_aware_grid()
    h = float(np.max(g["voxel"]))
    rng = np.random.default_rng(29)
    pts1 = rng.uniform(g["bmin"], g["bmax"], (30_000, 3)).astype(np.float32)
    pts2 = np.asarray(g["pts"], np.float32)
    for mode in modes:
        ref1 = grid.query_host(pts1, mode=mode)
        ref2 = grid.query_host(pts2, mode=mode)
        _close(_static(lib, grid, pts1, mode), ref1, h)
        _close(_static(lib, grid, pts2, mode), ref2, h)


def test_static_staging_allocates_nothing(cuda):
    """On a fresh handle, static-path calls (before any sdfo_query_host on it)
    leave the free device memory and the library's cached blocks unchanged.
    A first call on another handle is made beforehand: loading the library's
    kernels and the static array on first use is the driver's, once per
    process, and not what this checks."""
    import torch

    from sdfo import _native as N

    lib = N.load()
    warm, g = _grid()
    h = float(g["voxel"][0])
    rng = np.random.default_rng(31)
    pts1 = rng.uniform(g["bmin"], g["bmax"], (40_000, 3)).astype(np.float32)
    pts2 = rng.uniform(g["bmin"], g["bmax"], (10_000, 3)).astype(np.float64)
    for mode in (2, 3):
        _static(lib, warm, pts1, mode)
        _static(lib, warm, pts2, mode)
    fresh, _ = _grid()
    torch.cuda.synchronize()
    free0, held0 = torch.cuda.mem_get_info()[0], _held(lib)
    out = {mode: (_static(lib, fresh, pts1, mode), _static(lib, fresh, pts2, mode))
           for mode in (2, 3)}
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert _held(lib) == held0
    for mode in (2, 3):
        _close(out[mode][0], fresh.query_host(pts1, mode=mode), h)
        _close(out[mode][1], fresh.query_host(pts2, mode=mode), h)
