"""Backward-Euler contact steps (sdfo_be_stepper, sdfo/be.py) against
BackwardEulerIntegrator.step (prototype/src/integrators/implicit_be.py) run
by the prototype itself (tests/golden/be_steps.npz, make_golden.py) and
against its restatement (oracle/be_port.py), which is pinned to those
fixtures on the CPU."""
import ctypes

import numpy as np
import pytest

from conftest import golden

SCENES = ["flat_drop", "tilted_drop"]
# row layout of be_steps.npz: t, r(3), R(9), v(3), w(3), phase, dt_current,
# stable_count, release_count, min_dt_hits, last_gap, last_penetration,
# last_normal_velocity, last_toi, h (the step taken from this row)


def _scene_args(d, name):
    prm = d[name + "_params"]
    return dict(mass=prm[0], inertia=np.diag(prm[1:4]), k=prm[4], order=prm[5], damping=prm[6],
                mu=prm[7], reg=prm[8])


def _qb(d, phi=None):
    from oracle import interp_np

    spec = dict(bmin=d["bmin"], voxel=d["voxel"], shape=tuple(d["shape"]))
    phi = d["phi"] if phi is None else phi

    def qb(Y):
        gap, grad, valid, _ = interp_np.query(spec, phi, d["normal"], 2, Y)
        gn = np.linalg.norm(grad, axis=1)
        unit = np.zeros_like(grad)
        unit[:, 2] = 1.0
        ok = valid & (gn > 1e-30)
        unit[ok] = grad[ok] / gn[ok, None]
        return gap, grad, gn, unit, valid

    return qb


def _port_scene(d, name):
    from oracle import be_port as P

    a = _scene_args(d, name)
    w = d["quad_w"] / d["quad_w"].sum()
    return P.Scene(_qb(d), d["quad_x"], w, d["bmin"], d["bmax"], 0.01, a["k"], a["order"],
                   a["damping"], a["mu"], a["reg"], a["mass"], a["inertia"])


def _load_row(integ, row):
    from oracle import be_port as P

    st = P.BodyState(row[1:4].copy(), row[4:13].reshape(3, 3).copy(), row[13:16].copy(),
                     row[16:19].copy(), row[0])
    rg = integ.region
    rg.phase, rg.dt_current = int(row[19]), row[20]
    rg.stable_count, rg.release_count, rg.min_dt_hits = int(row[21]), int(row[22]), int(row[23])
    rg.last_gap, rg.last_penetration, rg.last_normal_velocity, rg.last_toi = row[24:28]
    return st


def _row_of(st, rg):
    return np.concatenate([[st.t], st.r, st.R.ravel(), st.v, st.w,
                           [rg.phase, rg.dt_current, rg.stable_count, rg.release_count,
                            rg.min_dt_hits, rg.last_gap, rg.last_penetration,
                            rg.last_normal_velocity, rg.last_toi]])


def _close(out, ref, tol, atol=1e-15):
    """Elementwise |out - ref| <= tol |ref| + atol (equal infinities pass)."""
    both_inf = np.isinf(out) & np.isinf(ref) & (np.sign(out) == np.sign(ref))
    o = np.where(both_inf, 0.0, out)
    r = np.where(both_inf, 0.0, ref)
    return np.all(np.abs(o - r) <= tol * np.abs(r) + atol)


@pytest.mark.parametrize("name", SCENES)
def test_port_steps_match_prototype(name):
    """Every recorded step of the prototype reproduced by the oracle from the
    recorded state before it (free flight, time-of-impact bisection,
    impact, active contact)."""
    from oracle import be_port as P

    d = golden("be_steps.npz")
    a = d[name]
    sc = _port_scene(d, name)
    phases = set()
    for k in range(len(a) - 1):
        integ = P.Integrator(sc)
        st = _load_row(integ, a[k])
        h = integ.step(st, 1e-3)
        assert h == a[k][28], k
        assert _close(_row_of(st, integ.region), a[k + 1][:28], 1e-12), k
        phases.add(int(a[k + 1][19]))
    assert {0, 2, 3} <= phases


def test_be_params_defaults():
    """sdfo_be_params_default = BackwardEulerIntegrator.__init__ defaults."""
    from oracle import be_port as P

    from sdfo import be

    p = be.default_params()
    q = P.Params()
    assert (p.max_iter, p.line_search, p.max_toi_bisect_iter, p.stable_steps, p.release_steps) == \
        (q.max_iter, int(q.line_search), q.max_toi_bisect_iter, q.stable_steps, q.release_steps)
    assert (p.tol, p.pen_max, p.dt_min, p.dt_impact, p.dt_contact, p.dt_max_contact, p.dt_normal,
            p.dt_growth) == (q.tol, q.pen_max, q.dt_min, q.dt_impact, q.dt_contact,
                             q.dt_max_contact, q.dt_normal, q.dt_growth)


def test_scene_layout_matches_the_c_struct():
    from sdfo import _native as N
    from sdfo import be

    class Scene(ctypes.Structure):
        _fields_ = [("body", N.BodyState), ("t", ctypes.c_double), ("dt_current", ctypes.c_double),
                    ("last_gap", ctypes.c_double), ("last_penetration", ctypes.c_double),
                    ("last_normal_velocity", ctypes.c_double), ("last_toi", ctypes.c_double),
                    ("phase", ctypes.c_int32), ("stable_count", ctypes.c_int32),
                    ("release_count", ctypes.c_int32), ("min_dt_hits", ctypes.c_int32)]

    assert ctypes.sizeof(Scene) == 8 * be.SCENE_DOUBLES
    s = Scene()
    body = N.BodyState()
    body.r[2] = 0.5
    p = be.default_params()
    N.load().sdfo_be_scene_init(ctypes.byref(s), ctypes.byref(body), 2.0, ctypes.byref(p))
    assert s.body.r[2] == 0.5 and s.t == 2.0 and s.dt_current == p.dt_normal
    assert np.isinf(s.last_gap) and np.isinf(s.last_toi) and s.phase == 0


# --------------------------------------------------------------------- GPU
def _stepper(d, name, max_scenes):
    from sdfo import SdfGrid
    from sdfo.be import BEStepper

    a = _scene_args(d, name)
    spec = dict(bmin=d["bmin"], bmax=d["bmax"], voxel=d["voxel"], shape=tuple(d["shape"]))
    grid = SdfGrid.from_dense(spec, d["phi"], d["normal"])
    st = BEStepper(grid, d["quad_x"], d["quad_w"], a["mass"], a["inertia"], a["k"], order=a["order"],
                   damping=a["damping"], friction=a["mu"], regularizer=a["reg"],
                   activation_distance=1e-5, narrow_margin=0.01, max_scenes=max_scenes)
    return grid, st


def _rows_to_scenes(st, rows):
    from sdfo.be import BEStepper

    dct = dict(t=rows[:, 0], r=rows[:, 1:4], R=rows[:, 4:13], v=rows[:, 13:16], w=rows[:, 16:19],
               phase=rows[:, 19], dt_current=rows[:, 20], stable_count=rows[:, 21],
               release_count=rows[:, 22], min_dt_hits=rows[:, 23], last_gap=rows[:, 24],
               last_penetration=rows[:, 25], last_normal_velocity=rows[:, 26], last_toi=rows[:, 27])
    return BEStepper.pack(dct)


def _scenes_to_rows(st, scenes):
    u = st.unpack(scenes)
    return np.concatenate([u["t"][:, None], u["r"], u["R"].reshape(-1, 9), u["v"], u["w"],
                           np.stack([u["phase"], u["dt_current"], u["stable_count"], u["release_count"],
                                     u["min_dt_hits"], u["last_gap"], u["last_penetration"],
                                     u["last_normal_velocity"], u["last_toi"]], axis=1)], axis=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", SCENES)
def test_gpu_steps_match_prototype(cuda, name):
    """Every recorded step of the prototype, all of them as scenes of one
    launch: the step taken, the phase and counters exactly; body state and
    region measurements within 1e-9 relative (FP64 throughout; the least
    squares solve and BLAS sums of the reference round differently)."""
    import torch

    d = golden("be_steps.npz")
    a = d[name]
    grid, st = _stepper(d, name, max_scenes=len(a))
    scenes = _rows_to_scenes(st, a[:-1])
    h = st.step(scenes, 1e-3)
    torch.cuda.synchronize()
    out = _scenes_to_rows(st, scenes)
    h = h.cpu().numpy()
    for k in range(len(a) - 1):
        ref = a[k + 1][:28]
        assert abs(h[k] - a[k][28]) <= 1e-12 * a[k][28], (k, h[k], a[k][28])
        assert out[k][19] == ref[19] and np.all(out[k][21:24] == ref[21:24]), (k, out[k][19:24], ref[19:24])
        assert _close(out[k], ref, 1e-9), (k, out[k] - ref)


@pytest.mark.gpu
def test_gpu_trajectories_match_port(cuda):
    """Eight scenes (random drops over the slab, both contact laws) advanced
    60 steps on the GPU and by the oracle: steps taken and phases equal,
    states within 1e-7 relative at the end."""
    import torch

    from oracle import be_port as P

    d = golden("be_steps.npz")
    rng = np.random.default_rng(7)
    for name in SCENES:
        grid, st = _stepper(d, name, max_scenes=8)
        sc = _port_scene(d, name)
        r = np.zeros((8, 3))
        R = np.zeros((8, 3, 3))
        for i in range(8):
            ax = rng.normal(size=3)
            ax /= np.linalg.norm(ax)
            ang = rng.uniform(0, 0.4)
            K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
            R[i] = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
            r[i] = [rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05),
                    -(R[i] @ d["quad_x"].T)[2].min() + rng.uniform(0.0005, 0.003)]
        v = np.column_stack([rng.normal(size=(8, 2)) * 0.05, -rng.uniform(0.05, 0.3, 8)])
        w = rng.normal(size=(8, 3)) * 0.5
        scenes = st.scenes(r, R, v, w)
        hs = []
        for _ in range(60):
            hs.append(st.step(scenes, 1e-3).cpu().numpy())
        torch.cuda.synchronize()
        out = _scenes_to_rows(st, scenes)
        for i in range(8):
            integ = P.Integrator(sc)
            s = P.BodyState(r[i].copy(), R[i].copy(), v[i].copy(), w[i].copy(), 0.0)
            for k in range(60):
                h = integ.step(s, 1e-3)
                assert abs(h - hs[k][i]) <= 1e-9 * h, (name, i, k, h, hs[k][i])
            ref = _row_of(s, integ.region)
            assert out[i][19] == ref[19], (name, i)
            assert _close(out[i][:19], ref[:19], 1e-7), (name, i, out[i][:19] - ref[:19])


@pytest.mark.gpu
def test_gpu_integrate_matches_port(cuda):
    """BEStepper.integrate (BackwardEulerIntegrator.integrate: steps of at most
    dt until t_end) for four scenes over 14 ms; the first, which meets the
    plane after about 13 ms (then steps of 10 us), against the oracle's own
    integrate loop."""
    from oracle import be_port as P

    d = golden("be_steps.npz")
    grid, st = _stepper(d, "flat_drop", max_scenes=4)
    r = np.array([[0.0, 0.0, 0.011], [0.01, 0.0, 0.02], [0.0, -0.02, 0.015], [0.0, 0.0, 0.05]])
    R = np.tile(np.eye(3), (4, 1, 1))
    v = np.tile([0.0, 0.0, -0.2], (4, 1))
    scenes = st.scenes(r, R, v=v)
    st.integrate(scenes, T=0.014, dt=1e-3)
    u = st.unpack(scenes)
    assert np.all(np.abs(u["t"] - 0.014) <= 1e-12)
    integ = P.Integrator(_port_scene(d, "flat_drop"))
    s = P.BodyState(r[0].copy(), R[0].copy(), v[0].copy(), np.zeros(3), 0.0)
    steps = 0
    while s.t < 0.014 - 1e-15:
        integ.step(s, min(1e-3, 0.014 - s.t))
        steps += 1
    assert steps > 50 and integ.region.phase == 3  # in contact, 10 us steps
    assert u["phase"][0] == integ.region.phase
    ref = np.concatenate([s.r, s.R.ravel(), s.v, s.w])
    out = np.concatenate([u["r"][0], u["R"][0].ravel(), u["v"][0], u["w"][0]])
    assert _close(out, ref, 1e-6, atol=1e-9), out - ref


@pytest.mark.gpu
@pytest.mark.parametrize("threads", [256, 32])
def test_gpu_advance_graph_matches_steps(cuda, threads):
    """sdfo_be_stepper_advance (integrate's steps replayed as one CUDA graph,
    each scene's step size min(dt, t_end - t) worked out on the device) gives
    the same states, bit for bit, as single steps whose sizes the host works
    out by implicit_be.py:121-122; the graph is replayed with the same
    arguments, and the unfinished count matches the host's."""
    import torch

    from sdfo import _native as N

    d = golden("be_steps.npz")
    grid, st = _stepper(d, "flat_drop", max_scenes=5)
    N.check(N.load().sdfo_be_stepper_set_threads(st._h, threads))
    r = np.array([[0.0, 0.0, 0.0115], [0.01, 0.0, 0.02], [0.0, -0.02, 0.012], [0.0, 0.0, 0.05],
                  [0.0, 0.0, 0.03]])
    R = np.tile(np.eye(3), (5, 1, 1))
    v = np.tile([0.0, 0.0, -0.2], (5, 1))
    a = st.scenes(r, R, v=v)
    b = a.clone()
    # scene 3 runs 2.5 ms, scene 4 is already at its end time
    t_end = a[:, 18] + torch.tensor([0.006, 0.006, 0.006, 0.0025, 0.0], dtype=torch.float64, device="cuda")
    unfinished = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        st.advance(a, t_end, 1e-3, launches=4, unfinished=unfinished)
    te = t_end.cpu().numpy()
    for _ in range(8):
        t = b[:, 18].cpu().numpy()
        req = np.where(t < te - 1e-15, np.minimum(1e-3, te - t), 0.0)
        st.step(b, torch.as_tensor(req, device="cuda"))
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    t = a[:, 18].cpu().numpy()
    assert int(unfinished.item()) == int(np.sum(t < te - 1e-15))
    assert t[4] == 0.0 and abs(t[3] - 0.0025) <= 1e-15


@pytest.mark.gpu
def test_gpu_threads_per_scene_agree(cuda):
    """One warp (32 threads), 128 and 256 threads per scene: the same steps
    (reductions summed in another order: states within 1e-12 relative)."""
    import torch

    d = golden("be_steps.npz")
    a = d["flat_drop"]
    outs = []
    for th in (256, 128, 32):
        grid, st = _stepper(d, "flat_drop", max_scenes=len(a))
        from sdfo import _native as N

        N.check(N.load().sdfo_be_stepper_set_threads(st._h, th))
        scenes = _rows_to_scenes(st, a[:-1])
        h = st.step(scenes, 1e-3)
        torch.cuda.synchronize()
        outs.append((h.cpu().numpy(), _scenes_to_rows(st, scenes)))
    for k in (1, 2):
        assert np.array_equal(outs[0][0], outs[k][0])
        assert _close(outs[0][1], outs[k][1], 1e-12, atol=1e-18)


def _port_scene_exact(d, name):
    from oracle import interp_np

    sc = _port_scene(d, name)
    spec = dict(bmin=d["bmin"], voxel=d["voxel"], shape=tuple(d["shape"]))
    sc.hess_batch = lambda Y: interp_np.trilinear_hessian(spec, d["phi"], Y)
    return sc


def _stepper_exact(d, name, max_scenes):
    from sdfo import SdfGrid
    from sdfo.be import BEStepper, default_params

    a = _scene_args(d, name)
    spec = dict(bmin=d["bmin"], bmax=d["bmax"], voxel=d["voxel"], shape=tuple(d["shape"]))
    grid = SdfGrid.from_dense(spec, d["phi"], d["normal"])
    st = BEStepper(grid, d["quad_x"], d["quad_w"], a["mass"], a["inertia"], a["k"], order=a["order"],
                   damping=a["damping"], friction=a["mu"], regularizer=a["reg"],
                   activation_distance=1e-5, narrow_margin=0.01, max_scenes=max_scenes,
                   params=default_params(tangent="exact"))
    return grid, st


@pytest.mark.gpu
@pytest.mark.parametrize("name", SCENES)
def test_gpu_exact_tangent_steps_match_port(cuda, name):
    """Exact-tangent mode (exact contact every residual, analytic dR/dV):
    every recorded state of the prototype stepped once on the GPU, all as
    scenes of one launch, against the restatement's exact Newton from the
    same state: the step taken and the phase and counters exactly, body
    state and region measurements within 1e-9 relative; the GPU's Newton
    iteration count equals the restatement's."""
    import torch

    from oracle import be_port as P

    d = golden("be_steps.npz")
    a = d[name]
    grid, st = _stepper_exact(d, name, max_scenes=len(a))
    scenes = _rows_to_scenes(st, a[:-1])
    st.stats(reset=True)
    h = st.step(scenes, 1e-3)
    torch.cuda.synchronize()
    stats = st.stats()
    out = _scenes_to_rows(st, scenes)
    h = h.cpu().numpy()
    sc = _port_scene_exact(d, name)
    iters = 0
    for k in range(len(a) - 1):
        integ = P.Integrator(sc, P.Params(tangent="exact"))
        s = _load_row(integ, a[k])
        hk = integ.step(s, 1e-3)
        iters += integ.newton_iterations
        ref = _row_of(s, integ.region)
        assert abs(h[k] - hk) <= 1e-12 * hk, (k, h[k], hk)
        assert out[k][19] == ref[19] and np.all(out[k][21:24] == ref[21:24]), (k, out[k][19:24], ref[19:24])
        assert _close(out[k], ref, 1e-9), (k, out[k] - ref)
    assert stats["newton_iterations"] == iters
    assert stats["be_solves"] >= len(a) - 1


@pytest.mark.gpu
def test_gpu_exact_tangent_trajectories_and_iterations(cuda):
    """Eight random drops per contact law advanced 60 steps in both tangent
    modes: the exact mode's trajectories against the restatement's exact
    Newton (steps and phases equal, states within 1e-7 relative) with no
    more Newton iterations than the reference mode; the three thread
    layouts give the same exact-mode states (to the last bits: they sum
    the points in different orders)."""
    import torch

    from oracle import be_port as P

    d = golden("be_steps.npz")
    rng = np.random.default_rng(11)
    for name in SCENES:
        r = np.zeros((8, 3))
        R = np.zeros((8, 3, 3))
        for i in range(8):
            ax = rng.normal(size=3)
            ax /= np.linalg.norm(ax)
            ang = rng.uniform(0, 0.4)
            K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
            R[i] = np.eye(3) + np.sin(ang) * K + (1 - np.cos(ang)) * K @ K
            r[i] = [rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05),
                    -(R[i] @ d["quad_x"].T)[2].min() + rng.uniform(0.0005, 0.003)]
        v = np.column_stack([rng.normal(size=(8, 2)) * 0.05, -rng.uniform(0.05, 0.3, 8)])
        w = rng.normal(size=(8, 3)) * 0.5
        runs = {}
        for mode, threads in (("exact", 256), ("exact", 128), ("exact", 32), ("reference", 256)):
            grid, st = (_stepper_exact(d, name, 8) if mode == "exact" else _stepper(d, name, 8))
            from sdfo import _native as N

            N.check(N.load().sdfo_be_stepper_set_threads(st._h, threads))
            scenes = st.scenes(r, R, v, w)
            hs = [st.step(scenes, 1e-3).cpu().numpy() for _ in range(60)]
            torch.cuda.synchronize()
            runs[(mode, threads)] = (_scenes_to_rows(st, scenes), hs, st.stats())
        ex, hs_ex, stats_ex = runs[("exact", 256)]
        for t in (128, 32):
            # the layouts sum the points in different orders: last bits only
            assert np.array_equal(runs[("exact", t)][0][:, 19], ex[:, 19]), t
            assert all(_close(runs[("exact", t)][0][i][:19], ex[i][:19], 1e-9) for i in range(8)), t
        rf, _, stats_rf = runs[("reference", 256)]
        assert stats_ex["newton_iterations"] <= stats_rf["newton_iterations"], (stats_ex, stats_rf)
        sc = _port_scene_exact(d, name)
        for i in range(8):
            integ = P.Integrator(sc, P.Params(tangent="exact"))
            s = P.BodyState(r[i].copy(), R[i].copy(), v[i].copy(), w[i].copy(), 0.0)
            for k in range(60):
                h = integ.step(s, 1e-3)
                assert abs(h - hs_ex[k][i]) <= 1e-9 * h, (name, i, k, h, hs_ex[k][i])
            ref = _row_of(s, integ.region)
            assert ex[i][19] == ref[19], (name, i)
            assert _close(ex[i][:19], ref[:19], 1e-7), (name, i, ex[i][:19] - ref[:19])
