"""sdfo_query_host with pinned buffers runs as a chunked three-stream
pipeline (copy-in on the caller's stream, query and copy-out on two streams
of the handle).  Its results must equal the device-buffer query bit for bit: the
chunks run the same kernels on the same points.  Covered: a remainder chunk
shorter than a CTA tile, growing chunks, more chunks than the pipeline keeps
events for (the last one takes the rest), float64 points, every optional
output, pageable buffers (single-shot path) and repeated calls on one
handle."""
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


def _pinned_query(lib, grid, pts, mode, outputs):
    import torch

    n = len(pts)
    hp = torch.from_numpy(pts).pin_memory()
    bufs = {"gap": torch.full((n,), np.nan).pin_memory()}
    for k in outputs:
        bufs[k] = (torch.full((n,), 7, dtype=torch.uint8) if k == "valid"
                   else torch.full((n, 3), np.nan)).pin_memory()
    P = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())  # noqa: E731
    from sdfo import _native as N

    N.check(lib.sdfo_query_host(grid.handle, mode, P(hp), 1 if pts.dtype == np.float64 else 0, n,
                                P(bufs["gap"]), P(bufs.get("grad")), P(bufs.get("unit")),
                                P(bufs.get("witness")), P(bufs.get("valid")), None))
    return {k: v.numpy() for k, v in bufs.items()}


def _device_query(grid, pts, mode, outputs):
    import torch

    x = torch.tensor(pts, device="cuda")
    out = grid.query_tensors(x, mode=mode, unit="unit" in outputs, witness="witness" in outputs,
                             valid=True)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("chunk,growth,n", [(4096, 130, 50_077), (4096, 100, 300_000),
                                             (256, 100, 1000), (32768, 200, 300_000)])
@pytest.mark.parametrize("outputs", [("grad", "valid"), ("grad", "unit", "witness", "valid")])
@pytest.mark.parametrize("out_mode", [1, 2, 3])
def test_pipelined_host_query_equals_device_query(cuda, chunk, growth, n, outputs, out_mode):
    from sdfo import _native as N

    lib = N.load()
    grid, g = _grid()
    rng = np.random.default_rng(n)
    pts = rng.uniform(g["bmin"], g["bmax"], (n, 3)).astype(np.float32)
    before = N.get_tuning()
    try:
        N.set_tuning(host_chunk_queries=chunk, host_chunk_growth_pct=growth, host_io_mode=out_mode)
        for mode in (2, 3):
            host = _pinned_query(lib, grid, pts, mode, outputs)
            dev = _device_query(grid, pts, mode, outputs)
            for k in ("gap",) + tuple(outputs):
                assert np.array_equal(host[k], dev[k]), (mode, k)
        # float64 points
        p64 = pts.astype(np.float64) + 1e-9
        host = _pinned_query(lib, grid, p64, 3, outputs)
        dev = _device_query(grid, p64, 3, outputs)
        for k in ("gap",) + tuple(outputs):
            assert np.array_equal(host[k], dev[k]), k
        # pageable buffers take the single-shot path: same results
        pg = grid.query_host(pts, mode=3)
        dev = _device_query(grid, pts, 3, ("grad", "unit", "witness", "valid"))
        for k in ("gap", "grad", "unit", "witness"):
            assert np.array_equal(pg[k], dev[k]), k
        assert np.array_equal(pg["valid"], dev["valid"].astype(bool))
    finally:
        N.set_tuning(**before)
