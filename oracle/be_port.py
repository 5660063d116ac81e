"""NumPy restatement of the prototype's implicit Backward-Euler contact step
for one free rigid body A against the SDF of a fixed body B (oracle).

TEST INFRASTRUCTURE ONLY.  Follows prototype/src/integrators/implicit_be.py
(BackwardEulerIntegrator) with one movable body, one contact pair and no
joints or drives, and the SDFContactEngine it drives
(prototype/src/dynamics/contacts_sdf.py), restated here with its culling
(oracle/point_bvh.py) and its linearisation cache:
  - step (implicit_be.py:131-181): initially penetrating regions become
    IMPACTING; h_cap = min(dt, cap of active regions); TOI search for
    inactive regions; the real step to the TOI or to h_cap; contact phase
    state machine (_refresh_contact_states, :248-295)
  - _find_earliest_new_contact / _bisect_toi_pair (:311-394): a trial BE step
    over h_cap, then bisection on [0, h] with BE trial steps (at most 60
    halvings, bracket width contact_dt_min)
  - _step_be (:468-505): Newton on the velocities V = (v, w) of body A with
    max_iter, tol on max |R|, the heuristic diagonal tangent
    (_contact_tangent / _tangent, :606-687), least squares solve and the
    backtracking line search (:689-697); the engine's linearisation cache is
    on while contact regions are active
  - _kinematic_update (:507-534): r = r0 + h v, R = exp([h w]x) R0 (Rodrigues)
  - _residual (:536-604): M (V - V0) / h + C - Q, M = diag(m I, R Ib R^T),
    C = w x (Iw w), Q = m g + contact (F_A, tau_A) of the allowed regions
  - the engine's cache (contacts_sdf.py:306-326): the first evaluation of a
    cached step queries the narrow-filtered points and stores (g, grad,
    valid) by position plus the SDF-frame translation; later evaluations with
    the same number of narrow-filtered points use g + grad . (t - t_ref),
    the stored gradient and validity.
The measure the in-residual `any_contact` flag takes (:592-601) is unused by
the reference and not restated.

Params.tangent = "exact" selects the exact Newton method that replaces the
reference's cache and heuristic tangent: every residual evaluates contact
exactly (no linearisation cache), and the tangent is the analytic Jacobian
dR/dV of the residual -- M/h, the derivatives of the rotational inertia and
gyroscopic terms through R(w), and the contact block dQ/dV = Jv + Jp
diag(h I, h J_l(h w)), where Jp is d(F, tau)/d(dx, dtheta) at fixed
velocities (R <- exp([dtheta]x) R), Jv is d(F, tau)/d(v, w) at a fixed pose,
and J_l is the left Jacobian of SO(3).  The per-point derivatives are the
force law's (contacts_sdf.py:329-385) differentiated by hand, with the
trilinear interpolant's Hessian (Scene.hess_batch).  `jacobians_fd` and
`tangent_fd` give the same matrices by central differences for the tests.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass, field

import numpy as np

from oracle import point_bvh as B

INACTIVE, APPROACHING, IMPACTING, ACTIVE, STABLE, LEAVING = 0, 1, 2, 3, 4, 5
ACTIVE_SET = (IMPACTING, ACTIVE, STABLE, LEAVING)


@dataclass
class Params:
    """BackwardEulerIntegrator.__init__ defaults (implicit_be.py:60-107)."""
    max_iter: int = 20
    tol: float = 1e-8
    line_search: bool = True
    pen_max: float = 1e-6
    dt_min: float = 1e-8
    dt_impact: float = 1e-7
    dt_contact: float = 1e-5
    dt_max_contact: float = 1e-4
    dt_normal: float = 1e-3
    dt_growth: float = 1.5
    stable_steps: int = 5
    release_steps: int = 3
    max_toi_bisect_iter: int = 60
    tangent: str = "reference"  # or "exact"

    @property
    def release_gap(self):
        return max(5.0 * self.pen_max, 1e-9)


@dataclass
class Region:
    """ContactRegionState (implicit_be.py:22-39)."""
    phase: int = INACTIVE
    dt_current: float = 1e-3
    stable_count: int = 0
    release_count: int = 0
    min_dt_hits: int = 0
    last_gap: float = np.inf
    last_penetration: float = 0.0
    last_normal_velocity: float = 0.0
    last_toi: float = np.inf


@dataclass
class BodyState:
    r: np.ndarray
    R: np.ndarray
    v: np.ndarray
    w: np.ndarray
    t: float = 0.0

    def copy(self):
        return BodyState(self.r.copy(), self.R.copy(), self.v.copy(), self.w.copy(), self.t)


@dataclass
class Scene:
    query_batch: object        # Y (N,3) -> (g, raw_grad, grad_norm, unit, valid)
    X: np.ndarray              # quadrature points, body A frame
    w: np.ndarray              # weights (normalised)
    bmin: np.ndarray
    bmax: np.ndarray
    narrow_margin: float
    k: float
    order: float
    damping: float
    mu: float
    regularizer: float
    mass: float
    inertia: np.ndarray        # body frame
    gravity: np.ndarray = field(default_factory=lambda: np.array([0.0, 0.0, -9.81]))
    rB: np.ndarray = field(default_factory=lambda: np.zeros(3))
    RB: np.ndarray = field(default_factory=lambda: np.eye(3))
    bvh: tuple = None
    hess_batch: object = None  # Y (N,3) -> (N,3,3) interpolant Hessian ("exact" tangent)

    def __post_init__(self):
        if self.bvh is None:
            self.bvh = B.build(self.X)


class Cache:
    def __init__(self):
        self.enabled = False
        self.cleared = True
        self.g = self.grad = self.valid = self.t_ref = None
        self.lactive_len = None


class Integrator:
    def __init__(self, scene: Scene, params: Params = None):
        self.s = scene
        self.p = params or Params()
        self.region = Region(dt_current=self.p.dt_normal)
        self.cache = Cache()
        self._M = None
        self._temp = None
        self.newton_iterations = 0

    # -------------------------------------------------------------- engine
    def _cull(self, st):
        return B.cull_indices(self.s.X, self.s.bvh, self.s.bmin, self.s.bmax, st.r, st.R,
                              self.s.narrow_margin)

    def evaluate(self, st, jac=False):
        """SDFContactEngine.evaluate (contacts_sdf.py:225-385) with the cache;
        with jac, also (Jp, Jv): the 6x6 Jacobians of (F, tau) w.r.t. the
        pose (dx, dtheta) and the velocities (v, w)."""
        s, c = self.s, self.cache
        idx = self._cull(st)
        R_sdf = s.RB.T @ st.R
        t_sdf = s.RB.T @ (st.r - s.rB)
        Y = (R_sdf @ s.X[idx].T + t_sdf[:, None]).T
        local = np.nonzero(np.abs(Y[:, 2]) < s.narrow_margin)[0]
        zero = (np.zeros(3), np.zeros(3)) + ((np.zeros((6, 6)), np.zeros((6, 6))) if jac else ())
        if len(local) == 0:
            return zero
        act_idx = idx[local]
        use = c.enabled and not c.cleared and c.lactive_len is not None and len(local) == c.lactive_len
        if use:
            g = c.g + c.grad @ (t_sdf - c.t_ref)
            raw = c.grad
            gn = np.linalg.norm(raw, axis=1)
            valid = c.valid
        else:
            g, raw, gn, _, valid = s.query_batch(Y[local])
            if c.enabled:
                c.g, c.grad, c.valid = g.copy(), raw.copy(), valid.copy()
                c.t_ref = t_sdf.copy()
                c.lactive_len = len(local)
                c.cleared = False
        p_all = s.k * np.maximum(-g, 0.0) ** s.order
        vm = valid & (p_all > 1e-30)
        if not np.any(vm):
            return zero
        gi = act_idx[vm]
        gv = g[vm]
        p = s.k * np.maximum(-gv, 0.0) ** s.order
        rg = (s.RB @ raw[vm].T).T
        gnv = gn[vm]
        xw = (st.r[:, None] + st.R @ s.X[gi].T).T
        wv = s.w[gi]
        off = xw - st.r[None, :]
        fn = p[:, None] * rg
        phat = p * gnv
        vB = np.zeros(3)
        wB = np.zeros(3)
        if s.damping > 0:
            uAd = st.v[None, :] + np.cross(st.w[None, :], off)
            uBd = vB[None, :] + np.cross(wB[None, :], xw - s.rB[None, :])
            vn = np.sum((uAd - uBd) * rg, axis=1)
            fn = fn + s.damping * (-vn)[:, None] * rg * (gv < 0.0)[:, None]
        uA = st.v[None, :] + np.cross(st.w[None, :], off)
        uB = vB[None, :] + np.cross(wB[None, :], xw - s.rB[None, :])
        u = uA - uB
        un = rg / np.maximum(gnv[:, None], 1e-30)
        ut = u - np.sum(u * un, axis=1, keepdims=True) * un
        den = np.sqrt(np.linalg.norm(ut, axis=1) ** 2 + s.regularizer ** 2)
        ft = np.zeros_like(fn)
        a = s.mu * phat > 0
        if np.any(a):
            ft[a] = -s.mu * phat[a, None] * ut[a] / den[a, None]
        fq = fn + ft
        F = np.sum(wv[:, None] * fq, axis=0)
        tau = np.sum(wv[:, None] * np.cross(off, fq), axis=0)
        if not jac:
            return F, tau
        Hs = s.hess_batch(Y[local][vm])
        Hw = np.einsum("ij,njk,lk->nil", s.RB, Hs, s.RB)
        dlt = -gv
        pp = -s.k * s.order * dlt ** (s.order - 1.0)      # dp/dg
        I3 = np.eye(3)[None]
        udn = np.sum(u * un, axis=1)
        P = I3 - un[:, :, None] * un[:, None, :]
        Mt = (I3 - ut[:, :, None] * ut[:, None, :] / den[:, None, None] ** 2) / den[:, None, None]
        fr = (s.mu * phat > 0).astype(float)[:, None, None]
        dm = 1.0 if s.damping > 0 else 0.0
        # dfq/dg, dfq/d(world gradient), dfq/du
        a_g = pp[:, None] * rg - fr[:, :, 0] * s.mu * (gnv * pp)[:, None] * ut / den[:, None]
        B = p[:, None, None] * I3 \
            - dm * s.damping * (rg[:, :, None] * u[:, None, :] + vn[:, None, None] * I3) \
            + fr * (-s.mu * p[:, None, None] * ut[:, :, None] * un[:, None, :] / den[:, None, None]
                    + s.mu * p[:, None, None] * Mt @ ((udn[:, None, None] * I3
                                                       + un[:, :, None] * u[:, None, :]) @ P))
        U = -dm * s.damping * rg[:, :, None] * rg[:, None, :] - fr * s.mu * phat[:, None, None] * (Mt @ P)
        G = a_g[:, :, None] * rg[:, None, :] + B @ Hw
        Gt = G - U @ _skew(wB)[None]
        Ox = _skew_n(off)
        Fx = _skew_n(fq)
        Wx = _skew(st.w)[None]
        Dth = -Gt @ Ox - U @ Wx @ Ox
        W = wv[:, None, None]
        Jp = np.zeros((6, 6))
        Jv = np.zeros((6, 6))
        Jp[:3, :3] = np.sum(W * Gt, 0)
        Jp[:3, 3:] = np.sum(W * Dth, 0)
        Jp[3:, :3] = np.sum(W * (Ox @ Gt), 0)
        Jp[3:, 3:] = np.sum(W * (Ox @ Dth + Fx @ Ox), 0)
        Jv[:3, :3] = np.sum(W * U, 0)
        Jv[:3, 3:] = np.sum(W * (-U @ Ox), 0)
        Jv[3:, :3] = np.sum(W * (Ox @ U), 0)
        Jv[3:, 3:] = np.sum(W * (-Ox @ U @ Ox), 0)
        return F, tau, Jp, Jv

    def jacobians_fd(self, st, hx=1e-8, hth=1e-8, hv=1e-6):
        """Central differences of evaluate (no cache): (Jp, Jv)."""
        Jp = np.zeros((6, 6))
        Jv = np.zeros((6, 6))

        def ev(q):
            F, t = self.evaluate(q)
            return np.concatenate([F, t])

        for k in range(6):
            a, b = st.copy(), st.copy()
            if k < 3:
                a.r[k] += hx
                b.r[k] -= hx
                Jp[:, k] = (ev(a) - ev(b)) / (2 * hx)
            else:
                e = np.zeros(3)
                e[k - 3] = hth
                a.R = _expm(e) @ st.R
                b.R = _expm(-e) @ st.R
                Jp[:, k] = (ev(a) - ev(b)) / (2 * hth)
            a, b = st.copy(), st.copy()
            (a.v if k < 3 else a.w)[k % 3] += hv
            (b.v if k < 3 else b.w)[k % 3] -= hv
            Jv[:, k] = (ev(a) - ev(b)) / (2 * hv)
        return Jp, Jv

    def measure(self, st):
        """measure_pair (contacts_sdf.py:171-214), uncached."""
        s = self.s
        m, _, _ = B.measure(s.query_batch, s.X, s.bvh, s.bmin, s.bmax, s.narrow_margin, st.r, st.R,
                            st.v, st.w, s.rB, s.RB, np.zeros(3), np.zeros(3))
        return m  # gap, penetration, normal_velocity, min_index, active_count, valid_count

    # ------------------------------------------------------------ dynamics
    @staticmethod
    def kinematic_update(q0, V, dt):
        st = q0.copy()
        st.v = V[:3].copy()
        st.w = V[3:6].copy()
        st.r = q0.r + dt * st.v
        dth = dt * st.w
        n = np.linalg.norm(dth)
        if n > 1e-30:
            a = dth / n
            c, s = np.cos(n), np.sin(n)
            dR = (c * np.eye(3) + s * np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
                  + (1 - c) * np.outer(a, a))
            st.R = dR @ q0.R
        else:
            st.R = q0.R.copy()
        return st

    def residual(self, z, q0, dt, allowed):
        s = self.s
        st = self.kinematic_update(q0, z, dt)
        self._temp = st
        Iw = st.R @ s.inertia @ st.R.T
        M = np.zeros((6, 6))
        M[:3, :3] = s.mass * np.eye(3)
        M[3:, 3:] = Iw
        C = np.zeros(6)
        C[3:] = np.cross(st.w, Iw @ st.w)
        Q = np.zeros(6)
        Q[:3] = s.mass * s.gravity
        if allowed:
            F, tau = self.evaluate(st)
            Q[:3] += F
            Q[3:] += tau
        V0 = np.concatenate([q0.v, q0.w])
        self._M = M
        return M @ (z - V0) / dt + C - Q

    def tangent_exact(self, z, q0, dt, allowed):
        """The analytic dR/dV at z (module docstring)."""
        s = self.s
        st = self.kinematic_update(q0, z, dt)
        Iw = st.R @ s.inertia @ st.R.T
        w = st.w
        dw = w - q0.w
        Jl = left_jacobian(dt * w)
        K = np.zeros((6, 6))
        K[:3, :3] = s.mass / dt * np.eye(3)
        K[3:, 3:] = Iw / dt + (-_skew(Iw @ dw) + Iw @ _skew(dw)) @ Jl
        K[3:, 3:] += -_skew(Iw @ w) + _skew(w) @ Iw + dt * _skew(w) @ (-_skew(Iw @ w) + Iw @ _skew(w)) @ Jl
        if allowed:
            _, _, Jp, Jv = self.evaluate(st, jac=True)
            T = np.zeros((6, 6))
            T[:3, :3] = dt * np.eye(3)
            T[3:, 3:] = dt * Jl
            K -= Jv + Jp @ T
        return K

    def tangent_fd(self, z, q0, dt, allowed, eps=1e-7):
        """Central differences of the residual (exact contact) in V."""
        K = np.zeros((6, 6))
        for i in range(6):
            zp, zm = z.copy(), z.copy()
            zp[i] += eps
            zm[i] -= eps
            K[:, i] = (self.residual(zp, q0, dt, allowed) - self.residual(zm, q0, dt, allowed)) / (2 * eps)
        return K

    def tangent(self, dt, allowed):
        s = self.s
        K = self._M / dt
        if allowed:
            area = np.sum(s.w)
            vel = np.linalg.norm(self._temp.v)
            d = max(vel * dt, 1e-10)
            if s.order == 1:
                stiff = s.k * dt
            else:
                stiff = s.k * s.order * (d ** (s.order - 1)) * dt + 5e2
            tot = stiff + s.damping * area
            for i in range(3):
                K[i, i] += tot
        return K

    def step_be(self, state, dt, allowed):
        """_step_be: state advanced in place; `allowed` = contact forces on."""
        q0 = state.copy()
        z = np.concatenate([q0.v, q0.w])
        exact = self.p.tangent == "exact"
        self.cache.enabled = allowed and not exact
        self.cache.cleared = True
        try:
            R = self.residual(z, q0, dt, allowed)
            for _ in range(self.p.max_iter):
                if np.max(np.abs(R)) < self.p.tol:
                    break
                self.newton_iterations += 1
                if exact:
                    dz = np.linalg.solve(self.tangent_exact(z, q0, dt, allowed), -R)
                else:
                    K = self.tangent(dt, allowed)
                    dz = np.linalg.lstsq(K, -R, rcond=1e-12)[0]
                alpha = 1.0
                if self.p.line_search:
                    r0 = np.linalg.norm(R)
                    alpha = 1.0
                    for a in (1.0, 0.5, 0.25, 0.125, 0.0625):
                        if np.linalg.norm(self.residual(z + a * dz, q0, dt, allowed)) < r0:
                            alpha = a
                            break
                z = z + alpha * dz
                R = self.residual(z, q0, dt, allowed)
            new = self.kinematic_update(q0, z, dt)
            state.r, state.R, state.v, state.w = new.r, new.R, new.v, new.w
            state.t = q0.t + dt
        finally:
            self.cache.enabled = False
            self.cache.cleared = True

    # ----------------------------------------------------- state machine
    def _active(self):
        return self.region.phase in ACTIVE_SET

    def _cap(self):
        return self.region.dt_current if self._active() else self.p.dt_normal

    def _store(self, m):
        rg = self.region
        rg.last_gap, rg.last_penetration, rg.last_normal_velocity = m[0], m[1], m[2]

    def _bisect(self, state, dt, allowed, m1):
        p = self.p
        lo, hi, hm, hit = 0.0, dt, m1, False
        for _ in range(p.max_toi_bisect_iter):
            if hi - lo <= p.dt_min:
                hit = True
                break
            mid = 0.5 * (lo + hi)
            tr = state.copy()
            self.step_be(tr, mid, allowed)
            m = self.measure(tr)
            if m[0] <= 0.0 or m[1] > p.pen_max:
                hi, hm = mid, m
            else:
                lo = mid
        if hi < p.dt_min and dt >= p.dt_min:
            hi, hit = p.dt_min, True
            tr = state.copy()
            self.step_be(tr, hi, allowed)
            hm = self.measure(tr)
        if hi <= 0.0:
            return None
        pen = 0.0 if hm is None else hm[1]
        if pen > p.pen_max and not hit:
            hi = max(lo, min(hi, p.dt_min))
            hit = True
        return min(hi, dt), pen, hit

    def step(self, state, dt):
        """BackwardEulerIntegrator.step: advances `state`, returns the step."""
        p, rg = self.p, self.region
        m = self.measure(state)  # _activate_initially_penetrating_regions
        self._store(m)
        if rg.phase == INACTIVE and m[0] <= 0.0:
            rg.phase = IMPACTING
            rg.dt_current = min(p.dt_impact, p.dt_contact)
        h_cap = min(dt, self._cap())
        event = None
        if rg.phase == INACTIVE and h_cap > 0:
            allowed = False  # the only region is inactive
            m0 = self.measure(state)
            tr = state.copy()
            self.step_be(tr, h_cap, allowed)
            m1 = self.measure(tr)
            if m0[0] > 0.0 and (m1[0] <= 0.0 or m1[1] > p.pen_max):
                event = self._bisect(state, h_cap, allowed, m1)
        if event is not None:
            toi, pen, hit = event
            self.step_be(state, toi, self._active())
            rg.phase = IMPACTING
            rg.dt_current = min(p.dt_impact, p.dt_contact)
            rg.last_toi = toi
            if hit:
                rg.min_dt_hits += 1
            self._store(self.measure(state))
            return toi
        self.step_be(state, h_cap, self._active())
        self._refresh(state)
        return h_cap

    def _refresh(self, state):
        p, rg = self.p, self.region
        m = self.measure(state)
        old = rg.last_penetration
        self._store(m)
        if rg.phase == INACTIVE:
            return
        if m[0] > p.release_gap and m[2] >= -1e-5:
            rg.release_count += 1
            rg.phase = LEAVING
            rg.dt_current = min(p.dt_normal, max(rg.dt_current * p.dt_growth, p.dt_contact))
            if rg.release_count >= p.release_steps:
                rg.phase, rg.dt_current = INACTIVE, p.dt_normal
                rg.stable_count = rg.release_count = rg.min_dt_hits = 0
                rg.last_toi = np.inf
            return
        rg.release_count = 0
        if rg.phase == IMPACTING:
            rg.phase = ACTIVE
            rg.dt_current = max(p.dt_contact, p.dt_min)
            return
        change = abs(m[1] - old)
        base = max(abs(old), p.pen_max)
        stable_pen = change <= p.pen_max or change / base <= 5e-2
        stable_vn = abs(m[2]) <= 1e-5
        if m[4] > 0 and stable_pen and stable_vn:
            rg.stable_count += 1
        else:
            rg.stable_count = 0
        if rg.stable_count >= p.stable_steps:
            rg.phase = STABLE
            rg.dt_current = min(p.dt_max_contact, p.dt_normal,
                                max(rg.dt_current * p.dt_growth, p.dt_contact))
        else:
            rg.phase = ACTIVE
            rg.dt_current = max(p.dt_contact, p.dt_min)


def _skew(a):
    return np.array([[0.0, -a[2], a[1]], [a[2], 0.0, -a[0]], [-a[1], a[0], 0.0]])


def _skew_n(a):
    S = np.zeros((len(a), 3, 3))
    S[:, 0, 1], S[:, 0, 2] = -a[:, 2], a[:, 1]
    S[:, 1, 0], S[:, 1, 2] = a[:, 2], -a[:, 0]
    S[:, 2, 0], S[:, 2, 1] = -a[:, 1], a[:, 0]
    return S


def _expm(phi):
    n = np.linalg.norm(phi)
    if n < 1e-300:
        return np.eye(3)
    K = _skew(phi / n)
    return np.eye(3) + np.sin(n) * K + (1 - np.cos(n)) * K @ K


def left_jacobian(phi):
    """J_l(phi) of SO(3): exp(phi + d) = exp([J_l(phi) d]x) exp(phi) + O(d^2)."""
    t = np.linalg.norm(phi)
    S = _skew(phi)
    if t < 1e-4:
        a = 0.5 - t * t / 24.0
        b = 1.0 / 6.0 - t * t / 120.0
    else:
        a = (1.0 - np.cos(t)) / (t * t)
        b = (t - np.sin(t)) / (t * t * t)
    return np.eye(3) + a * S + b * S @ S


def clone(integ: Integrator) -> Integrator:
    out = Integrator(integ.s, integ.p)
    out.region = copy.deepcopy(integ.region)
    return out
