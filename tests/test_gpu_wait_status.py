"""Bounded waits of the bulk-copy pipelines (the dense forward with the walk
kernel off, and the saved backward) run out without faulting or hanging, set
their status bits, and the synchronous host entry points turn them into
SDFO_ERR_DEVICE_STATUS instead of returning partial results.

The wait is made to run out through the test-only sdfo_debug_wait_test:
every CTA skips the bulk load of its first tile (so that tile's mbarrier
never completes) and the main-loop wait gives up after 1000 try-wait
iterations.  The kernels then wait for the loads they did issue and return;
the context stays usable, which the last part checks by querying again."""
import ctypes

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

ERR_DEVICE_STATUS = -5


def _grid():
    from sdfo import SdfGrid

    g = golden("dense_torus.npz")
    spec = dict(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    return SdfGrid.from_dense(spec, g["phi"], g["normal"], g["hessian"]), g


def _status(lib, clear):
    f = ctypes.c_uint32(0)
    from sdfo import _native as N

    N.check(lib.sdfo_device_status(ctypes.byref(f), 1 if clear else 0))
    return int(f.value)


def test_waits_run_out_and_are_reported(cuda):
    import torch

    from sdfo import _native as N

    lib = N.load()
    grid, g = _grid()
    rng = np.random.default_rng(3)
    n = 4096 * 3 + 17
    pts = rng.uniform(g["bmin"], g["bmax"], (n, 3)).astype(np.float32)
    x = torch.tensor(pts, device="cuda")
    ref = grid.query_tensors(x, mode=3)
    torch.cuda.synchronize()
    ref = {k: v.cpu().numpy() for k, v in ref.items()}
    _status(lib, clear=True)
    p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
    before = N.get_tuning()
    try:
        # the dense forwards on the bulk-copy pipeline (the walk kernel, the
        # default, has no bounded wait)
        N.set_tuning(query_walk=1)
        N.check(lib.sdfo_debug_wait_test(1000, 1))
        # device path: the call is asynchronous and succeeds; the word
        # records the abort of the pipelined forward (bit 1)
        grid.query_tensors(x, mode=3)
        torch.cuda.synchronize()
        assert _status(lib, clear=True) & 2
        # host paths: the abort is an error, and the word is cleared
        gap = np.zeros(n, np.float32)
        grad = np.zeros((n, 3), np.float32)
        valid = np.zeros(n, np.uint8)
        rc = lib.sdfo_query_host(grid.handle, 3, p(pts), 0, n, p(gap), p(grad), None, None,
                                 p(valid), None)
        assert rc == ERR_DEVICE_STATUS
        assert "bounded wait" in N.last_error()
        assert _status(lib, clear=False) == 0
        rc = lib.sdfo_query_host_static(grid.handle, 3, p(pts), 0, n, p(gap), p(grad), p(valid),
                                        None)
        assert rc == ERR_DEVICE_STATUS
        assert _status(lib, clear=False) == 0
        # saved-linearisation backward for points: bit 0
        gap_d = torch.empty(n, device="cuda")
        grad_d = torch.empty((n, 3), device="cuda")
        valid_d = torch.empty(n, dtype=torch.uint8, device="cuda")
        hess6 = torch.zeros((n, 6), device="cuda")
        dgap = torch.ones(n, device="cuda")
        dpts = torch.empty((n, 3), device="cuda")
        P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        N.check(lib.sdfo_query_linearize(grid.handle, 3, P(x), n, P(gap_d), P(grad_d),
                                         P(valid_d), P(hess6), None))
        N.check(lib.sdfo_query_backward_saved(grid.handle, 3, P(x), n, P(grad_d), P(hess6),
                                              P(valid_d), P(dgap), None, P(dpts), None, None))
        torch.cuda.synchronize()
        f = _status(lib, clear=True)
        assert f & 1 and f & 2
    finally:
        N.check(lib.sdfo_debug_wait_test(0, 0))
        N.set_tuning(**before)
        _status(lib, clear=True)
    # normal operation again: the same results as before, no status
    out = grid.query_host(pts, mode=3)
    assert np.array_equal(out["gap"], ref["gap"])
    assert np.array_equal(out["grad"], ref["grad"])
    assert np.array_equal(out["valid"], ref["valid"].astype(bool))
    assert _status(lib, clear=False) == 0
