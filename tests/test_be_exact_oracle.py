"""The exact Newton tangent of the BE restatement (oracle/be_port.py,
Params.tangent = "exact") pinned on the CPU:
* the hand-derived contact Jacobians -- d(F, tau)/d(dx, dtheta) at fixed
  velocities and d(F, tau)/d(v, w) at a fixed pose -- against central
  differences of SDFContactEngine.evaluate (restated, no cache) at states of
  the prototype's own recorded steps in contact, for both contact laws;
* the full analytic dR/dV against central differences of the residual;
* over 160 steps from the first recorded state, exact Newton reaches the
  same trajectory as the reference's cached, heuristic-tangent method (the
  cache is a first-order approximation inside each step, so the two agree
  to the Newton tolerance's order, not bit for bit) with fewer Newton
  iterations.
The GPU kernel's exact mode is checked against this restatement in
tests/test_be_step.py."""
import numpy as np
import pytest

from conftest import golden

SCENES = ["flat_drop", "tilted_drop"]


def _scene(d, name):
    from oracle import be_port as P
    from oracle import interp_np

    prm = d[name + "_params"]
    spec = dict(bmin=d["bmin"], voxel=d["voxel"], shape=tuple(d["shape"]))

    def qb(Y):
        gap, grad, valid, _ = interp_np.query(spec, d["phi"], d["normal"], 2, Y)
        gn = np.linalg.norm(grad, axis=1)
        unit = np.zeros_like(grad)
        unit[:, 2] = 1.0
        ok = valid & (gn > 1e-30)
        unit[ok] = grad[ok] / gn[ok, None]
        return gap, grad, gn, unit, valid

    w = d["quad_w"] / d["quad_w"].sum()
    return P.Scene(qb, d["quad_x"], w, d["bmin"], d["bmax"], 0.01, prm[4], prm[5], prm[6], prm[7],
                   prm[8], prm[0], np.diag(prm[1:4]),
                   hess_batch=lambda Y: interp_np.trilinear_hessian(spec, d["phi"], Y))


def _state(row):
    from oracle import be_port as P

    return P.BodyState(row[1:4].copy(), row[4:13].reshape(3, 3).copy(), row[13:16].copy(),
                       row[16:19].copy(), row[0])


@pytest.mark.parametrize("name", SCENES)
def test_contact_jacobians_match_central_differences(name):
    from oracle import be_port as P

    d = golden("be_steps.npz")
    integ = P.Integrator(_scene(d, name), P.Params(tangent="exact"))
    rows = d[name]
    checked = 0
    for k in range(0, len(rows), 13):
        st = _state(rows[k])
        F, tau, Jp, Jv = integ.evaluate(st, jac=True)
        if not np.any(F):
            continue
        Jp_fd, Jv_fd = integ.jacobians_fd(st)
        assert np.abs(Jp - Jp_fd).max() <= 1e-6 * np.abs(Jp_fd).max(), k
        assert np.abs(Jv - Jv_fd).max() <= 1e-6 * np.abs(Jv_fd).max(), k
        checked += 1
    assert checked >= 5


@pytest.mark.parametrize("name", SCENES)
def test_exact_tangent_matches_central_differences(name):
    from oracle import be_port as P

    d = golden("be_steps.npz")
    integ = P.Integrator(_scene(d, name), P.Params(tangent="exact"))
    rows = d[name]
    for k in (40, 90, 150):
        q0 = _state(rows[k])
        z = np.concatenate([q0.v, q0.w]) * 0.98 + 1e-3
        for h in (1e-5, 1e-4):
            K = integ.tangent_exact(z, q0, h, True)
            Kfd = integ.tangent_fd(z, q0, h, True)
            assert np.abs(K - Kfd).max() <= 1e-6 * np.abs(Kfd).max(), (k, h)
            # the contact block alone (M/h dominates the full matrix)
            K0 = integ.tangent_exact(z, q0, h, False)
            Kc, Kcfd = K - K0, Kfd - integ.tangent_fd(z, q0, h, False)
            assert np.abs(Kc - Kcfd).max() <= 1e-5 * np.abs(Kcfd).max(), (k, h)


@pytest.mark.parametrize("name", SCENES)
def test_exact_newton_same_trajectory_fewer_iterations(name):
    from oracle import be_port as P

    d = golden("be_steps.npz")
    out = {}
    for mode in ("reference", "exact"):
        integ = P.Integrator(_scene(d, name), P.Params(tangent=mode))
        st = _state(d[name][0])
        hs = [integ.step(st, 1e-3) for _ in range(160)]
        out[mode] = (integ.newton_iterations, st, hs, integ.region.phase)
    (n_ref, s_ref, h_ref, ph_ref), (n_ex, s_ex, h_ex, ph_ex) = out["reference"], out["exact"]
    assert h_ref == h_ex and ph_ref == ph_ex
    assert np.abs(s_ref.r - s_ex.r).max() <= 1e-9
    assert np.abs(s_ref.v - s_ex.v).max() <= 1e-5 * np.abs(s_ref.v).max()
    assert n_ex < n_ref
