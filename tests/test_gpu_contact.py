"""Fused contact kernel (sdfo_contact_eval) against the contact oracle.

Forces/torques: the oracle (oracle/contact_port.py, pinned to the
prototype's SDFContactEngine.evaluate) evaluated in FP64 on the same FP32
grid payload; tolerance 1e-5 of the pose's force (torque) magnitude.
Jacobian: central differences (h = 1e-7 m / 1e-6 rad) of the oracle with the
active point set, the damping switch (g < 0) and each point's interpolation
cell frozen at the base pose, i.e. the derivative of the smooth piece that
forward-mode AD differentiates (the damping switch is a step at g = 0 and the
trilinear gradient jumps across cell faces: unfrozen differences across
either are not derivatives); tolerance 1e-4 of the Jacobian's magnitude."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ring_cube(cuda):
    from sdfo import SdfGrid
    from sdfo import workloads as W

    c = W.c3_ring_cube(n_poses=4096)
    cv, ct = c["cube"]
    grid = SdfGrid.build_dense(cv, ct, **c["build"])
    d = grid.export_dense()
    spec = dict(bmin=grid.bmin, voxel=grid.voxel, shape=grid.shape)
    phi32 = d["phi"].astype(np.float32).astype(np.float64)
    n32 = d["normal"].astype(np.float32).astype(np.float64)
    return c, grid, spec, phi32, n32


def _oracle_eval(spec, phi, nrm, mode, c, i, r=None, R=None, freeze=None):
    from oracle import contact_port as cp
    from oracle import interp_np

    frozen_cells = None if freeze is None else freeze[1]

    def qb(Y):
        g, grad, valid, cells = interp_np.query(spec, phi, nrm, mode, Y, frozen_cells)
        qb.cells = cells
        return g, grad, np.linalg.norm(grad, axis=1), None, valid

    prm = c["params"]
    w = c["quad_w"] / c["quad_w"].sum()
    F, tau, g, mask = cp.evaluate_pose(
        qb, c["quad_x"], w, c["r"][i] if r is None else r, c["R"][i] if R is None else R,
        c["v"][i], c["w"][i], np.zeros(3), np.eye(3), np.zeros(3), np.zeros(3),
        prm["stiffness"], prm["order"], prm["damping"], prm["friction"], prm["regularizer"],
        freeze=None if freeze is None else freeze[0])
    return np.concatenate([F, tau]), mask, qb.cells


def _batch(grid, c, mode):
    from sdfo.contact import ContactBatch

    return ContactBatch(grid, c["quad_x"], c["quad_w"], mode=mode, **c["params"])


def _states(c, idx):
    from sdfo.contact import pack_states

    return pack_states(c["r"][idx], c["R"][idx], c["v"][idx], c["w"][idx])


def _body_b():
    from sdfo.contact import pack_states

    return pack_states(np.zeros((1, 3)), np.eye(3)[None])[0]


@pytest.mark.parametrize("mode", [2, 3])
def test_contact_forces_vs_oracle(ring_cube, mode):
    c, grid, spec, phi, nrm = ring_cube
    idx = np.arange(0, 4096, 97)
    ft = _batch(grid, c, mode).evaluate(_states(c, idx), _body_b()).cpu().numpy()
    n_contact = 0
    for k, i in enumerate(idx):
        ref, mask, _ = _oracle_eval(spec, phi, nrm, mode, c, i)
        sf = max(np.abs(ref[:3]).max(), 1e-6)
        st = max(np.abs(ref[3:]).max(), 1e-9)
        assert np.abs(ft[k, :3] - ref[:3]).max() <= 1e-5 * sf, (i, ft[k], ref)
        assert np.abs(ft[k, 3:] - ref[3:]).max() <= 1e-5 * st + 1e-5 * sf * 1e-3, (i, ft[k], ref)
        n_contact += bool(mask.any())
    assert n_contact >= 5


@pytest.mark.parametrize("mode", [2, 3])
def test_contact_jacobian_vs_frozen_fd(ring_cube, mode):
    from oracle.contact_port import rotvec

    c, grid, spec, phi, nrm = ring_cube
    # the 8 lowest poses that the oracle finds in contact, plus the two highest
    order = np.argsort(c["r"][:, 2])
    touching = []
    for i in order[:400]:
        if _oracle_eval(spec, phi, nrm, mode, c, i)[1].any():
            touching.append(int(i))
            if len(touching) == 8:
                break
    assert len(touching) == 8
    idx = np.array(touching + [int(order[-1]), int(order[-2])])
    ft, jac = _batch(grid, c, mode).evaluate(_states(c, idx), _body_b(), jacobian=True)
    jac = jac.cpu().numpy()
    errs = []
    for k, i in enumerate(idx):
        base, mask, cells = _oracle_eval(spec, phi, nrm, mode, c, i)
        if not mask.any():
            assert np.all(jac[k] == 0)
            continue
        J = np.zeros((6, 6))
        for j in range(6):
            cols = []
            for s in (1.0, -1.0):
                r, R = c["r"][i].copy(), c["R"][i].copy()
                if j < 3:
                    r[j] += s * 1e-7
                    h = 1e-7
                else:
                    th = np.zeros(3)
                    th[j - 3] = s * 1e-6
                    R = rotvec(th) @ R
                    h = 1e-6
                f, _, _ = _oracle_eval(spec, phi, nrm, mode, c, i, r, R, freeze=(mask, cells))
                cols.append(f)
            J[:, j] = (cols[0] - cols[1]) / (2 * h)
        scale = np.abs(J).max()
        err = np.abs(jac[k] - J).max() / scale
        errs.append(err)
        assert err <= 1e-4, (i, err)
    assert len(errs) >= 8


def test_fd_baseline_runs(ring_cube):
    """The forward-only finite-difference baseline (12 extra evaluations)."""
    from sdfo.contact import fd_jacobian

    c, grid, spec, phi, nrm = ring_cube
    idx = np.arange(0, 4096, 128)
    b = _batch(grid, c, 3)
    ft, jac = fd_jacobian(b, _states(c, idx), _body_b())
    ft2, jac2 = b.evaluate(_states(c, idx), _body_b(), jacobian=True)
    assert np.array_equal(ft.cpu().numpy(), ft2.cpu().numpy())
    assert jac.shape == jac2.shape == (len(idx), 6, 6)



def test_contact_force_autograd(ring_cube):
    """contact_force: dL/dr = J_x^T dL/dft and dL/dtheta = J_l(theta)^T
    J_theta^T dL/dft, with J_l checked against central differences of
    log(exp(theta + e) exp(theta)^-1) (scipy), at rotated poses in contact."""
    import torch
    from scipy.spatial.transform import Rotation

    from sdfo.contact import contact_force, so3_left_jacobian

    c, grid, spec, phi, nrm = ring_cube
    cb = _batch(grid, c, 2)
    order = np.argsort(c["r"][:, 2])
    idx = []
    for i in order[:400]:
        if _oracle_eval(spec, phi, nrm, 2, c, i)[1].any():
            idx.append(int(i))
            if len(idx) == 6:
                break
    idx = np.array(idx)
    P = len(idx)
    dev = "cuda"
    theta0 = np.random.default_rng(3).normal(size=(P, 3)) * 0.2
    # R0 = exp(-[theta0]) R so that the pose rotation exp([theta0]) R0 is R
    R0 = torch.tensor(np.einsum("pij,pjk->pik", Rotation.from_rotvec(-theta0).as_matrix(),
                                c["R"][idx]), device=dev)
    r = torch.tensor(c["r"][idx], dtype=torch.float64, device=dev, requires_grad=True)
    theta = torch.tensor(theta0, dtype=torch.float64, device=dev, requires_grad=True)
    v = torch.tensor(c["v"][idx], device=dev)
    w = torch.tensor(c["w"][idx], device=dev)
    ft = contact_force(cb, r, theta, R0, v, w, _body_b())
    up = torch.randn_like(ft)
    (ft * up).sum().backward()
    _, jac = cb.evaluate(_states(c, idx), _body_b(), jacobian=True)
    g = torch.einsum("pi,pij->pj", up, jac)
    scale = float(g.abs().max())
    assert float((r.grad - g[:, :3]).abs().max()) <= 1e-9 * scale
    Jl = so3_left_jacobian(torch.tensor(theta0, device=dev)).cpu().numpy()
    for p in range(P):
        num = np.zeros((3, 3))
        base = Rotation.from_rotvec(theta0[p])
        for k in range(3):
            e = np.zeros(3)
            e[k] = 1e-6
            dp = (Rotation.from_rotvec(theta0[p] + e) * base.inv()).as_rotvec()
            dm = (Rotation.from_rotvec(theta0[p] - e) * base.inv()).as_rotvec()
            num[:, k] = (dp - dm) / 2e-6
        assert np.abs(num - Jl[p]).max() <= 1e-8
    want = torch.einsum("pij,pi->pj", torch.tensor(Jl, device=dev), g[:, 3:])
    assert float((theta.grad - want).abs().max()) <= 1e-9 * scale
