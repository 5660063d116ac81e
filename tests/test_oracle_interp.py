"""Pins the NumPy interpolant restatement (oracle/interp_np.py) to the C
restatement, and the contact oracle's finite-difference Jacobian to itself
(frozen-cell differences converge)."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("mode", [2, 3])
def test_interp_np_matches_port(port, mode):
    from oracle import interp_np

    g = golden("dense_torus.npz")
    spec = port.GridSpec(bmin=g["bmin"], bmax=g["bmax"], voxel=g["voxel"], shape=tuple(g["shape"]))
    q = port.query_dense(spec, g["phi"], g["normal"], None, mode, g["pts"])
    gap, grad, valid, _ = interp_np.query(spec, g["phi"], g["normal"], mode, g["pts"])
    assert np.array_equal(valid, q["valid"])
    h = float(g["voxel"][0])
    assert np.allclose(gap, q["gap"], rtol=1e-12, atol=1e-14 * h)
    assert np.allclose(grad, q["grad"], rtol=1e-10, atol=1e-12)


def test_frozen_cell_fd_matches_analytic_gradient(port):
    """Central differences of the frozen-cell interpolant reproduce the
    analytic gradient (the oracle the GPU Jacobians are checked with)."""
    from oracle import interp_np

    g = golden("dense_torus.npz")
    spec = dict(bmin=g["bmin"], voxel=g["voxel"], shape=tuple(g["shape"]))
    pts = g["pts"]
    gap, grad, valid, cells = interp_np.query(spec, g["phi"], g["normal"], 3, pts)
    hstep = 1e-7
    for a in range(3):
        e = np.zeros(3)
        e[a] = hstep
        gp, _, _, _ = interp_np.query(spec, g["phi"], g["normal"], 3, pts + e, cells)
        gm, _, _, _ = interp_np.query(spec, g["phi"], g["normal"], 3, pts - e, cells)
        fd = (gp - gm) / (2 * hstep)
        assert np.allclose(fd[valid], grad[valid, a], rtol=1e-5, atol=1e-6)
