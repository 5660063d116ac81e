"""Batched penalty contact between a quadrature body A and the SDF of body B.

``ContactBatch.evaluate`` runs the fused kernel (sdfo_contact_eval): for every
pose of A it evaluates SDFContactEngine.evaluate's law
(prototype/src/dynamics/contacts_sdf.py:296-385) over all quadrature points
and returns the total force / torque on A, optionally with the 6x6 Jacobian
d(F_A, tau_A)/d(dx, dtheta) (r_A += dx, R_A = exp([dtheta]x) R_A).

``fd_jacobian`` is the finite-difference baseline the analytic Jacobian
replaces: 12 extra forward evaluations per pose (central differences).

Body states are float64 CUDA tensors of shape (P, 18) laid out as
sdfo_body_state: r (3), R row-major (9), v (3), w (3).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native as N
from .grid import _stream_ptr, _t_ptr


def pack_states(r, R, v=None, w=None, device="cuda") -> torch.Tensor:
    """(P,3) r, (P,3,3) R, (P,3) v, (P,3) w -> (P,18) float64 CUDA tensor."""
    r = torch.as_tensor(np.asarray(r, np.float64)).reshape(-1, 3)
    P = r.shape[0]
    R = torch.as_tensor(np.asarray(R, np.float64)).reshape(P, 9)
    v = torch.zeros(P, 3, dtype=torch.float64) if v is None else torch.as_tensor(
        np.asarray(v, np.float64)).reshape(P, 3)
    w = torch.zeros(P, 3, dtype=torch.float64) if w is None else torch.as_tensor(
        np.asarray(w, np.float64)).reshape(P, 3)
    return torch.cat([r, R, v, w], dim=1).contiguous().to(device)


def rotvec_to_matrix(theta: torch.Tensor) -> torch.Tensor:
    """Rodrigues: exp([theta]x) for (P,3) rotation vectors (float64)."""
    ang = torch.linalg.norm(theta, dim=1, keepdim=True)
    safe = torch.where(ang > 0, ang, torch.ones_like(ang))
    k = theta / safe
    K = torch.zeros(theta.shape[0], 3, 3, dtype=theta.dtype, device=theta.device)
    K[:, 0, 1], K[:, 0, 2] = -k[:, 2], k[:, 1]
    K[:, 1, 0], K[:, 1, 2] = k[:, 2], -k[:, 0]
    K[:, 2, 0], K[:, 2, 1] = -k[:, 1], k[:, 0]
    s = torch.sin(ang)[:, :, None]
    c = torch.cos(ang)[:, :, None]
    I = torch.eye(3, dtype=theta.dtype, device=theta.device).expand_as(K)
    return I + s * K + (1 - c) * (K @ K)


class ContactBatch:
    """Quadrature set of body A + contact parameters, bound to body B's grid.

    ``narrow_margin`` None evaluates every quadrature point.  A number applies
    SDFContactEngine's culling with that narrow margin (register_pair's
    default is 0.01): the point-BVH cull (AABB_BVH, ``leaf_size`` points per
    leaf) against body B's grid box with margin max(narrow_margin, 0.05),
    then evaluate's |Y_z| < narrow_margin filter (contacts_sdf.py:244-298);
    ``measure`` then applies the BVH cull as measure_pair does."""

    def __init__(self, grid, quad_x, quad_w, stiffness, order=1.0, damping=0.0, friction=0.5,
                 regularizer=1e-6, activation_distance=0.0, mode=N.TRILINEAR,
                 normalize_weights=True, narrow_margin=None, leaf_size=16, device="cuda"):
        self.grid = grid
        qx = np.ascontiguousarray(quad_x, np.float64).reshape(-1, 3)
        qw = np.ascontiguousarray(quad_w, np.float64).reshape(-1)
        if normalize_weights and qw.sum() > 1e-30:
            qw = qw / qw.sum()  # register_pair (contacts_sdf.py:52-56)
        self._qx64, self._qw64 = qx, qw
        self.narrow_margin = narrow_margin
        self.leaf_size = int(leaf_size)
        self._pair = None
        self.qx = torch.as_tensor(qx, dtype=torch.float32, device=device).contiguous()
        self.qw = torch.as_tensor(qw, dtype=torch.float32, device=device).contiguous()
        self.nq = qx.shape[0]
        self.params = N.ContactParams(float(stiffness), float(order), float(damping),
                                      float(friction), float(regularizer),
                                      float(activation_distance))
        self.mode = N.mode_id(mode)
        if self.mode not in (N.TRILINEAR, N.TRICUBIC):
            raise ValueError("contact supports Trilinear and Tricubic")
        if narrow_margin is not None:
            self._pair = self._make_pair(float(narrow_margin))

    def _make_pair(self, narrow_margin):
        out = ctypes.c_void_p()
        N.check(N.load().sdfo_contact_pair_create(
            self.grid.handle, self._qx64.ctypes.data_as(ctypes.c_void_p),
            self._qw64.ctypes.data_as(ctypes.c_void_p), self.nq, 0, narrow_margin, self.leaf_size,
            ctypes.byref(out)))
        return out

    def close(self):
        if getattr(self, "_pair", None) is not None and self._pair.value:
            N.load().sdfo_contact_pair_destroy(self._pair)
            self._pair = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _states(poses_a, body_b):
        pa = poses_a.contiguous()
        pb = body_b.reshape(18).contiguous()
        if pa.dtype != torch.float64 or pb.dtype != torch.float64:
            raise ValueError("body states must be float64")
        return pa, pb

    def evaluate(self, poses_a: torch.Tensor, body_b: torch.Tensor, jacobian=False,
                 out=None, stream=None):
        """poses_a (P,18), body_b (18,) float64 CUDA -> ft (P,6) [, jac (P,6,6)]."""
        pa, pb = self._states(poses_a, body_b)
        P = pa.shape[0]
        if out is None:
            ft = torch.empty((P, 6), dtype=torch.float64, device=pa.device)
            jac = torch.empty((P, 6, 6), dtype=torch.float64, device=pa.device) if jacobian else None
        else:
            ft, jac = out
        if self._pair is None:
            N.check(N.load().sdfo_contact_eval(self.grid.handle, self.mode, _t_ptr(self.qx),
                                               _t_ptr(self.qw), self.nq, _t_ptr(pa), P, _t_ptr(pb),
                                               ctypes.byref(self.params), _t_ptr(ft), _t_ptr(jac),
                                               _stream_ptr(stream)))
        else:
            N.check(N.load().sdfo_contact_pair_eval(self._pair, self.mode, _t_ptr(pa), P, _t_ptr(pb),
                                                    ctypes.byref(self.params), _t_ptr(ft),
                                                    _t_ptr(jac), None, _stream_ptr(stream)))
        return (ft, jac) if jacobian else ft

    def measure(self, poses_a: torch.Tensor, body_b: torch.Tensor, stream=None) -> dict:
        """measure_pair (contacts_sdf.py:171-214) per pose: dict of CUDA
        tensors gap, penetration, normal_velocity (float64), min_point_index,
        active_count, valid_count (int32)."""
        pa, pb = self._states(poses_a, body_b)
        if self._pair is None:
            self._pair = self._make_pair(-1.0)
        P = pa.shape[0]
        buf = torch.empty((P, 5), dtype=torch.float64, device=pa.device)
        N.check(N.load().sdfo_contact_pair_eval(self._pair, self.mode, _t_ptr(pa), P, _t_ptr(pb),
                                                ctypes.byref(self.params), None, None, _t_ptr(buf),
                                                _stream_ptr(stream)))
        ints = buf[:, 3:5].contiguous().view(torch.int32)
        return dict(gap=buf[:, 0], penetration=buf[:, 1], normal_velocity=buf[:, 2],
                    min_point_index=ints[:, 0], active_count=ints[:, 1], valid_count=ints[:, 2])


def perturbed_poses(poses: torch.Tensor, h_lin=1e-7, h_ang=1e-6) -> torch.Tensor:
    """The 12 central-difference pose batches: (12, P, 18), order
    +x, -x, +y, -y, +z, -z, +thx, -thx, ... ."""
    P = poses.shape[0]
    out = poses.unsqueeze(0).repeat(12, 1, 1)
    R = poses[:, 3:12].reshape(P, 3, 3)
    for a in range(3):
        for s, sign in enumerate((1.0, -1.0)):
            out[2 * a + s, :, a] += sign * h_lin
            th = torch.zeros(P, 3, dtype=poses.dtype, device=poses.device)
            th[:, a] = sign * h_ang
            out[6 + 2 * a + s, :, 3:12] = (rotvec_to_matrix(th) @ R).reshape(P, 9)
    return out


def fd_jacobian(batch: ContactBatch, poses: torch.Tensor, body_b: torch.Tensor, h_lin=1e-7,
                h_ang=1e-6):
    """Forward-only baseline: F(pose) plus 12 perturbed evaluations -> (ft, jac)."""
    ft = batch.evaluate(poses, body_b)
    pert = perturbed_poses(poses, h_lin, h_ang)
    P = poses.shape[0]
    fts = batch.evaluate(pert.reshape(12 * P, 18), body_b).reshape(12, P, 6)
    h = torch.tensor([h_lin] * 3 + [h_ang] * 3, dtype=torch.float64, device=poses.device)
    jac = (fts[0::2] - fts[1::2]) / (2.0 * h[:, None, None])  # (6 params, P, 6 outputs)
    return ft, jac.permute(1, 2, 0).contiguous()


def so3_left_jacobian(theta: torch.Tensor) -> torch.Tensor:
    """J_l(theta) of exp: exp([theta + d]x) = exp([J_l d]x) exp([theta]x) to
    first order; (P,3) -> (P,3,3), I + (1 - cos a)/a^2 K + (a - sin a)/a^3 K^2
    with K = [theta]x, a = |theta| (series below 1e-4)."""
    a = torch.linalg.norm(theta, dim=1)
    K = torch.zeros(theta.shape[0], 3, 3, dtype=theta.dtype, device=theta.device)
    K[:, 0, 1], K[:, 0, 2] = -theta[:, 2], theta[:, 1]
    K[:, 1, 0], K[:, 1, 2] = theta[:, 2], -theta[:, 0]
    K[:, 2, 0], K[:, 2, 1] = -theta[:, 1], theta[:, 0]
    small = a < 1e-4
    safe = torch.where(small, torch.ones_like(a), a)
    c1 = torch.where(small, 0.5 - a * a / 24.0, (1.0 - torch.cos(safe)) / (safe * safe))
    c2 = torch.where(small, 1.0 / 6.0 - a * a / 120.0, (safe - torch.sin(safe)) / (safe ** 3))
    I = torch.eye(3, dtype=theta.dtype, device=theta.device).expand_as(K)
    return I + c1[:, None, None] * K + c2[:, None, None] * (K @ K)


class ContactForce(torch.autograd.Function):
    """(F_A, tau_A) of a ContactBatch as a differentiable function of body A's
    position r (P,3) and a rotation vector theta (P,3), R = exp([theta]x) R0.
    The backward uses the kernel's analytic 6x6 Jacobian (forward mode, per
    quadrature point): dL/dr = J_x^T dL/dft, dL/dtheta = J_l(theta)^T
    J_theta^T dL/dft.  No reference counterpart (the reference tangent is a
    finite difference, implicit_be.py:661-687)."""

    @staticmethod
    def forward(ctx, r, theta, R0, v, w, body_b, batch):
        P = r.shape[0]
        R = rotvec_to_matrix(theta.detach()) @ R0
        poses = torch.cat([r.detach(), R.reshape(P, 9), v, w], dim=1).contiguous()
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            ft, jac = batch.evaluate(poses, body_b, jacobian=True)
            ctx.save_for_backward(theta.detach(), jac)
        else:
            ft = batch.evaluate(poses, body_b)
            ctx.save_for_backward(theta.detach(), None)
        return ft

    @staticmethod
    def backward(ctx, dft):
        theta, jac = ctx.saved_tensors
        g = torch.einsum("pi,pij->pj", dft.to(jac.dtype), jac)
        dr = g[:, :3] if ctx.needs_input_grad[0] else None
        dth = None
        if ctx.needs_input_grad[1]:
            dth = torch.einsum("pij,pi->pj", so3_left_jacobian(theta), g[:, 3:])
        return dr, dth, None, None, None, None, None


def contact_force(batch: ContactBatch, r, theta, R0, v, w, body_b):
    """Differentiable (F_A, tau_A) (P,6): see ContactForce."""
    return ContactForce.apply(r, theta, R0, v, w, body_b, batch)
