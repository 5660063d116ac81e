"""Batched Backward-Euler contact steps on the GPU (sdfo_be_stepper).

``BEStepper`` runs BackwardEulerIntegrator.step
(prototype/src/integrators/implicit_be.py:131-181) for many independent
scenes at once: each scene is one free rigid body A carrying a quadrature
set, against a fixed body B carrying a dense SDF grid, with
SDFContactEngine's culling and linearisation cache
(prototype/src/dynamics/contacts_sdf.py).  One CUDA thread block advances
one scene through its whole adaptive step -- time-of-impact bisection with
trial BE solves, Newton iterations with line search, the contact phase state
machine -- so a step of every scene is one kernel launch, and integrate's
steps replay as CUDA graphs of such launches.

Scenes live in a float64 CUDA tensor (n, 26) laid out as sdfo_be_scene:
r (3), R row-major (9), v (3), w (3), t, dt_current, last_gap,
last_penetration, last_normal_velocity, last_toi, then four int32 (phase,
stable_count, release_count, min_dt_hits) in the last two slots.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as N
from .contact import ContactBatch
from .grid import _stream_ptr, _t_ptr

SCENE_DOUBLES = 26
INACTIVE, IMPACTING, ACTIVE, STABLE, LEAVING = 0, 2, 3, 4, 5
PHASE_NAMES = {0: "INACTIVE", 1: "APPROACHING", 2: "IMPACTING", 3: "ACTIVE", 4: "STABLE",
               5: "LEAVING"}


TANGENTS = {"reference": N.BE_TANGENT_REFERENCE, "exact": N.BE_TANGENT_EXACT}


def default_params(**overrides) -> N.BEParams:
    """BackwardEulerIntegrator's defaults (implicit_be.py:60-107), with
    keyword overrides by field name (max_iter, tol, pen_max, dt_min, ...).
    tangent: "reference" (the reference's linearisation cache and diagonal
    tangent) or "exact" (exact contact every residual, analytic dR/dV)."""
    p = N.BEParams()
    N.load().sdfo_be_params_default(ctypes.byref(p))
    if isinstance(overrides.get("tangent"), str):
        overrides["tangent"] = TANGENTS[overrides["tangent"]]
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise ValueError(f"unknown BE parameter {k!r}")
        setattr(p, k, v)
    return p


class BEStepper:
    """A batch of scenes sharing body A's quadrature set and mass properties,
    body B's grid and pose, the contact law and the integrator parameters."""

    def __init__(self, grid, quad_x, quad_w, mass, inertia, stiffness, order=1, damping=0.0,
                 friction=0.5, regularizer=1e-6, activation_distance=0.0, narrow_margin=0.01,
                 gravity=(0.0, 0.0, -9.81), body_b=None, params=None, max_scenes=1024,
                 leaf_size=16, threads=256):
        self.contact = ContactBatch(grid, quad_x, quad_w, stiffness, order=order, damping=damping,
                                    friction=friction, regularizer=regularizer,
                                    activation_distance=activation_distance, mode=N.TRILINEAR,
                                    narrow_margin=-1.0 if narrow_margin is None else narrow_margin,
                                    leaf_size=leaf_size)
        self.params = params if params is not None else default_params()
        body = N.RigidBody()
        body.mass = float(mass)
        I = np.asarray(inertia, np.float64).reshape(3, 3)
        for k in range(9):
            body.inertia[k] = float(I.reshape(-1)[k])
        for k in range(3):
            body.gravity[k] = float(gravity[k])
        self.body = body
        bb = N.BodyState()
        rB, RB = (np.zeros(3), np.eye(3)) if body_b is None else (np.asarray(body_b[0], float),
                                                                    np.asarray(body_b[1], float))
        for k in range(3):
            bb.r[k] = float(rB[k])
        for k in range(9):
            bb.R[k] = float(RB.reshape(-1)[k])
        self.body_b = bb
        self.max_scenes = int(max_scenes)
        out = ctypes.c_void_p()
        N.check(N.load().sdfo_be_stepper_create(self.contact._pair, ctypes.byref(self.contact.params),
                                                ctypes.byref(self.body), ctypes.byref(self.body_b),
                                                ctypes.byref(self.params), self.max_scenes,
                                                ctypes.byref(out)))
        self._h = out
        N.check(N.load().sdfo_be_stepper_set_threads(self._h, int(threads)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.load().sdfo_be_stepper_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------- scenes
    def scenes(self, r, R, v=None, w=None, t=0.0, device="cuda") -> torch.Tensor:
        """Scenes at rest in the state machine (INACTIVE, dt_current =
        dt_normal, last_gap = last_toi = inf): (n, 26) float64 CUDA tensor."""
        r = np.asarray(r, np.float64).reshape(-1, 3)
        n = len(r)
        R = np.asarray(R, np.float64).reshape(n, 9)
        v = np.zeros((n, 3)) if v is None else np.asarray(v, np.float64).reshape(n, 3)
        w = np.zeros((n, 3)) if w is None else np.asarray(w, np.float64).reshape(n, 3)
        out = np.zeros((n, SCENE_DOUBLES))
        out[:, 0:3], out[:, 3:12], out[:, 12:15], out[:, 15:18] = r, R, v, w
        out[:, 18] = t
        out[:, 19] = self.params.dt_normal
        out[:, 20] = np.inf
        out[:, 23] = np.inf
        return torch.as_tensor(out).to(device).contiguous()

    @staticmethod
    def unpack(scenes: torch.Tensor) -> dict:
        """Scene tensor -> dict of numpy arrays (r, R, v, w, t, dt_current,
        last_gap, last_penetration, last_normal_velocity, last_toi, phase,
        stable_count, release_count, min_dt_hits)."""
        a = scenes.detach().cpu().numpy()
        ints = a[:, 24:26].copy().view(np.int32).reshape(-1, 4)
        return dict(r=a[:, 0:3], R=a[:, 3:12].reshape(-1, 3, 3), v=a[:, 12:15], w=a[:, 15:18],
                    t=a[:, 18], dt_current=a[:, 19], last_gap=a[:, 20], last_penetration=a[:, 21],
                    last_normal_velocity=a[:, 22], last_toi=a[:, 23], phase=ints[:, 0],
                    stable_count=ints[:, 1], release_count=ints[:, 2], min_dt_hits=ints[:, 3])

    @staticmethod
    def pack(d: dict, device="cuda") -> torch.Tensor:
        """Inverse of unpack (every key required)."""
        n = len(d["t"])
        a = np.zeros((n, SCENE_DOUBLES))
        a[:, 0:3], a[:, 3:12] = d["r"], np.asarray(d["R"]).reshape(n, 9)
        a[:, 12:15], a[:, 15:18], a[:, 18] = d["v"], d["w"], d["t"]
        a[:, 19], a[:, 20], a[:, 21] = d["dt_current"], d["last_gap"], d["last_penetration"]
        a[:, 22], a[:, 23] = d["last_normal_velocity"], d["last_toi"]
        ints = np.stack([d["phase"], d["stable_count"], d["release_count"], d["min_dt_hits"]],
                        axis=1).astype(np.int32)
        a[:, 24:26] = ints.view(np.float64).reshape(n, 2)
        return torch.as_tensor(a).to(device).contiguous()

    # ------------------------------------------------------------ stepping
    def step(self, scenes: torch.Tensor, dt, out_h=None, stream=None) -> torch.Tensor:
        """One BackwardEulerIntegrator.step of every scene (in place); dt a
        float or an (n,) float64 CUDA tensor (<= 0 leaves a scene as it is).
        Returns the step each scene took."""
        self._check(scenes)
        n = scenes.shape[0]
        if not torch.is_tensor(dt):
            dt = torch.full((n,), float(dt), dtype=torch.float64, device=scenes.device)
        dt = dt.contiguous()
        h = out_h if out_h is not None else torch.empty(n, dtype=torch.float64, device=scenes.device)
        N.check(N.load().sdfo_be_stepper_step(self._h, _t_ptr(scenes), n, _t_ptr(dt), _t_ptr(h),
                                              _stream_ptr(stream)))
        return h

    def advance(self, scenes: torch.Tensor, t_end: torch.Tensor, dt: float, launches: int = 8,
                unfinished: torch.Tensor = None, stream=None) -> None:
        """`launches` steps of BackwardEulerIntegrator.integrate's loop
        (implicit_be.py:121-127) for every scene short of its t_end (an (n,)
        float64 CUDA tensor), replayed as one CUDA graph.  `unfinished` (a
        one-element int32 CUDA tensor) receives the number of scenes still
        short of t_end.  Asynchronous."""
        self._check(scenes)
        t_end = self._t_end(scenes, t_end)
        if unfinished is not None and (unfinished.dtype != torch.int32 or unfinished.numel() < 1):
            raise ValueError("unfinished must be an int32 CUDA tensor")
        N.check(N.load().sdfo_be_stepper_advance(
            self._h, _t_ptr(scenes), scenes.shape[0], _t_ptr(t_end), float(dt), int(launches),
            _t_ptr(unfinished) if unfinished is not None else None, _stream_ptr(stream)))

    def integrate(self, scenes: torch.Tensor, T: float, dt: float, check_every=8, max_launches=100000,
                  stream=None) -> int:
        """BackwardEulerIntegrator.integrate (implicit_be.py:113-129) for every
        scene: steps of at most dt until each scene's t reaches its start
        time + T.  The steps run as CUDA graphs of `check_every` launches
        with a 4-byte read of the unfinished count after each.  Returns the
        number of launches; raises if max_launches ran out first."""
        self._check(scenes)
        t_end = (scenes[:, 18] + T).contiguous()
        made = ctypes.c_int64(0)
        left = ctypes.c_int32(0)
        N.check(N.load().sdfo_be_stepper_integrate(
            self._h, _t_ptr(scenes), scenes.shape[0], _t_ptr(t_end), float(dt), int(check_every),
            int(max_launches), ctypes.byref(made), ctypes.byref(left), _stream_ptr(stream)))
        if left.value:
            raise RuntimeError(f"{left.value} scenes short of their end time after {made.value} launches")
        return made.value

    def stats(self, reset=False) -> dict:
        """Newton iterations, residual evaluations and BE solves of every
        launch since creation or the last reset (synchronises the device)."""
        out = (ctypes.c_uint64 * 3)()
        N.check(N.load().sdfo_be_stepper_stats(self._h, out, 1 if reset else 0))
        return {"newton_iterations": int(out[0]), "residual_evaluations": int(out[1]),
                "be_solves": int(out[2])}

    @staticmethod
    def _check(scenes):
        if scenes.dtype != torch.float64 or scenes.dim() != 2 or scenes.shape[1] != SCENE_DOUBLES \
                or not scenes.is_contiguous() or not scenes.is_cuda:
            raise ValueError("scenes must be a contiguous (n, 26) float64 CUDA tensor")

    @staticmethod
    def _t_end(scenes, t_end):
        if not torch.is_tensor(t_end) or t_end.dtype != torch.float64 or t_end.numel() != scenes.shape[0] \
                or not t_end.is_cuda:
            raise ValueError("t_end must be an (n,) float64 CUDA tensor")
        return t_end.contiguous()
