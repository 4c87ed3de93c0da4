"""Gradients of full-IPC rollouts by the adjoint method, with
checkpoint-and-recompute, and a torch.autograd.Function over them.

A rollout steps nxd_ipc_step (implicit Euler, the primitive-pair barrier).
Each step solves G(x; z) = 0 for x = (p, theta); its adjoint (nxd_ipc_adjoint,
the implicit function theorem at the converged x*) maps x_bar = dL/dx* to
the adjoints of the step's inputs.  This module chains the steps:

  outputs  p1 = x_p,  v1 = (x_p - p0) / dt,  w1 = x_theta / dt,
           q1 = Exp(x_theta) q0  (tangent adjoints: left rotations psi)
  x_bar_p     = p1_bar + v1_bar / dt
  x_bar_theta = w1_bar / dt + J_l(x_theta)^T psi1_bar
  p0_bar      = -v1_bar / dt + phat_bar        (phat = p0 + dt v0)
  v0_bar      = dt phat_bar
  w0_bar      = dt thetahat_bar                (thetahat = dt w0)
  psi0_bar    = Exp(x_theta)^T psi1_bar + phi_bar
and sums the parameter adjoints (masses, inertias, fixed-joint stiffnesses)
over the steps.  The forward pass keeps the state every `checkpoint_every`
steps; the backward pass re-steps each segment from its checkpoint to get
the segment's start states and converged iterates, then runs its adjoints
in reverse.  The reference has no adjoint; its parameter-identification
workflow (tools/compare_with_reference.py:85-165) differentiates by
re-simulation.

Supported scenes: bodies and fixed joints (FixedJoint), no control forms,
implicit Euler (nxd_ipc_adjoint's limits).
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional

import numpy as np

from . import abi


def _skew(v):
    return np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])


def _jr_c12(a):
    if a < 1e-2:
        a2 = a * a
        return 0.5 - a2 / 24.0 + a2 * a2 / 720.0, 1.0 / 6.0 - a2 / 120.0 + a2 * a2 / 5040.0
    return (1 - np.cos(a)) / (a * a), (a - np.sin(a)) / (a ** 3)


def exp_mat(th):
    """Exp(theta) as a rotation matrix."""
    a = np.linalg.norm(th)
    S = _skew(th)
    c1, _ = _jr_c12(a)
    sinc = 1.0 - a * a / 6.0 + a ** 4 / 120.0 if a < 1e-2 else np.sin(a) / a
    return np.eye(3) + sinc * S + c1 * S @ S


def left_jacobian(th):
    """J_l(theta): Exp(theta + d) = Exp(J_l d) Exp(theta) to first order."""
    c1, c2 = _jr_c12(np.linalg.norm(th))
    S = _skew(th)
    return np.eye(3) + c1 * S + c2 * S @ S


def quat_tangent_adjoint(q, qbar):
    """Left-tangent adjoint psi_bar of a quaternion q (w, x, y, z) from the
    4-vector gradient qbar: (d(Exp(psi) q)/dpsi at 0)^T qbar."""
    q = np.asarray(q, dtype=np.float64)
    qbar = np.asarray(qbar, dtype=np.float64)
    w, v = q[..., :1], q[..., 1:]
    return 0.5 * (w * qbar[..., 1:] + np.cross(v, qbar[..., 1:]) - qbar[..., :1] * v)


def iterate_of(state1: dict, dt: float) -> np.ndarray:
    """The converged iterate x* (6N) of the step that produced state1."""
    n = state1["position"].shape[0]
    x = np.zeros((n, 6))
    x[:, :3] = state1["position"]
    x[:, 3:] = state1["angular_velocity"] * dt
    return x.reshape(-1)


def _copy_state(st: dict) -> dict:
    return {k: np.array(v, dtype=np.float64, copy=True) for k, v in st.items()}


class IpcRollout:
    """A full-IPC rollout of `scene` on the device with adjoint gradients.

    step_fn(ctx) / adjoint_fn(ctx, start, x_star, x_bar) default to the
    device (runtime.Context.ipc_step / ipc_adjoint)."""

    def __init__(self, scene, params=None, checkpoint_every: int = 10, ctx=None,
                 adjoint_fn: Optional[Callable] = None, stream: Optional[int] = None):
        from . import runtime
        self.scene = scene
        self.params = params if params is not None else abi.ipc_params()
        self.k = max(1, int(checkpoint_every))
        self.ctx = ctx if ctx is not None else runtime.Context(scene)
        if stream:
            # its own CUDA stream (raw cudaStream_t), so that rollouts on other
            # host threads overlap on the device
            import ctypes
            runtime.lib().nxd_set_stream(self.ctx.h, ctypes.c_void_p(stream))
        self.adjoint_fn = adjoint_fn or (lambda start, xs, xb: self.ctx.ipc_adjoint(start, xs, xb, self.params))
        self.checkpoints = []
        self.steps = 0
        self.stats = []

    def _step(self):
        st = self.ctx.ipc_step(self.params)
        self.stats.append(st)
        return st

    def forward(self, steps: int) -> dict:
        """Steps from the scene's initial state; returns the final state."""
        self.ctx.set_state(self.scene.initial_state())
        self.checkpoints = []
        self.stats = []
        self.steps = steps
        for t in range(steps):
            if t % self.k == 0:
                self.checkpoints.append(_copy_state(self.ctx.state()))
            self._step()
        self.final = _copy_state(self.ctx.state())
        return self.final

    def backward(self, p_bar, q_bar=None, v_bar=None, w_bar=None) -> dict:
        """Adjoints of the initial state and the parameters for output
        adjoints of the final state: p_bar (N, 3), q_bar (N, 4) Euclidean
        gradients of the final orientations, v_bar / w_bar (N, 3)."""
        sc = self.scene
        n, nj, dt = sc.n_bodies, len(sc.joint_type), sc.dt
        T = self.final
        pb = np.array(p_bar, dtype=np.float64).reshape(n, 3)
        psib = (quat_tangent_adjoint(T["orientation"], np.asarray(q_bar, dtype=np.float64).reshape(n, 4))
                if q_bar is not None else np.zeros((n, 3)))
        vb = np.zeros((n, 3)) if v_bar is None else np.array(v_bar, dtype=np.float64).reshape(n, 3)
        wb = np.zeros((n, 3)) if w_bar is None else np.array(w_bar, dtype=np.float64).reshape(n, 3)
        mass_bar = np.zeros(n)
        inertia_bar = np.zeros((n, 3, 3))
        mu_bar = np.zeros(nj)
        friction_bar = 0.0
        for seg in range(len(self.checkpoints) - 1, -1, -1):
            t0 = seg * self.k
            t1 = min(self.steps, t0 + self.k)
            # recompute the segment: start states and the state after each step
            self.ctx.set_state(self.checkpoints[seg])
            starts, ends = [], []
            for _ in range(t0, t1):
                starts.append(_copy_state(self.ctx.state()))
                self.ctx.ipc_step(self.params)
                ends.append(_copy_state(self.ctx.state()))
            for t in range(len(starts) - 1, -1, -1):
                xs = iterate_of(ends[t], dt)
                th = xs.reshape(n, 6)[:, 3:]
                xbar = np.zeros((n, 6))
                xbar[:, :3] = pb + vb / dt
                xbar[:, 3:] = wb / dt + np.einsum("bji,bj->bi", np.array([left_jacobian(a) for a in th]), psib)
                r = self.adjoint_fn(starts[t], xs, xbar.reshape(-1))
                # the start positions enter through p^ = p0 + dt v0 and, with
                # friction, through the pairs frozen at the step start
                pb = -vb / dt + r["phat_bar"] + r.get("p0_bar", 0.0)
                vb = dt * r["phat_bar"]
                wb = dt * r["thetahat_bar"]
                psib = np.einsum("bji,bj->bi", np.array([exp_mat(a) for a in th]), psib) + r["phi_bar"]
                mass_bar += r["mass_bar"]
                inertia_bar += r["inertia_bar"]
                mu_bar += r["joint_mu_bar"]
                friction_bar += r.get("friction_mu_bar", 0.0)
        return {"position": pb, "orientation_tangent": psib, "velocity": vb, "angular_velocity": wb,
                "mass": mass_bar, "inertia": inertia_bar, "joint_stiffness": mu_bar, "friction": friction_bar}


def with_parameters(scene, velocity=None, mass=None, joint_stiffness=None, angular_velocity=None):
    """A copy of `scene` with the given initial velocities, masses and joint
    stiffnesses."""
    new = dataclasses.replace(scene, velocity=np.array(scene.velocity, dtype=np.float64, copy=True),
                              angular_velocity=np.array(scene.angular_velocity, dtype=np.float64, copy=True),
                              mass=np.array(scene.mass, dtype=np.float64, copy=True),
                              joint_stiffness=np.array(scene.joint_stiffness, dtype=np.float64, copy=True))
    if velocity is not None:
        new.velocity[...] = velocity
    if angular_velocity is not None:
        new.angular_velocity[...] = angular_velocity
    if mass is not None:
        new.mass[...] = mass
    if joint_stiffness is not None:
        new.joint_stiffness[...] = joint_stiffness
    return new


def make_rollout_function(stream: Optional[int] = None):
    """torch.autograd.Function: (velocity (N,3), mass (N), joint_stiffness
    (J), friction coefficient (scalar, or None: params.mu)) -> final poses
    (N, 7: position, orientation w x y z) of a full-IPC rollout, with the
    adjoint backward (the coefficient's gradient needs params with one
    lagging pass).  With `stream` (a raw cudaStream_t) the rollout's context
    issues its work there, so that several parameter sets run concurrently
    from host threads.  Built lazily so that importing this module does not
    import torch."""
    import torch

    class IpcRolloutFunction(torch.autograd.Function):
        @staticmethod
        def forward(fctx, velocity, mass, joint_stiffness, scene, params, steps, checkpoint_every, friction=None):
            sc = with_parameters(scene, velocity=velocity.detach().cpu().numpy(), mass=mass.detach().cpu().numpy(),
                                 joint_stiffness=joint_stiffness.detach().cpu().numpy())
            if friction is not None:
                params = abi.NxdIpcParams.from_buffer_copy(params)
                params.mu = float(friction.detach().cpu())
            fctx.has_friction = friction is not None
            r = IpcRollout(sc, params, checkpoint_every, stream=stream)
            st = r.forward(int(steps))
            fctx.rollout = r
            out = np.concatenate([st["position"], st["orientation"]], axis=1)
            return torch.as_tensor(out, dtype=torch.float64)

        @staticmethod
        def backward(fctx, grad):
            g = grad.detach().cpu().numpy()
            r = fctx.rollout
            b = r.backward(g[:, :3], g[:, 3:])
            dev = grad.device
            to = lambda a: torch.as_tensor(np.asarray(a), dtype=torch.float64, device=dev)
            gf = to(b["friction"]) if fctx.has_friction else None
            return to(b["velocity"]), to(b["mass"]), to(b["joint_stiffness"]), None, None, None, None, gf

    return IpcRolloutFunction
