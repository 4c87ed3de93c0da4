"""Differentiable rollouts of the contact step: Jacobians of a rollout's final
poses with respect to scene parameters, by central differences over copies of
the scene stepped together as one batch on the device (nxd_batch_*), and a
torch.autograd.Function over them.

This is a finite-difference gradient, not an adjoint.  The step it
differentiates is the reference's IPCSolver::step as written: ALM iterations
with hardening decisions, friction normal forces lagged by one ALM iteration,
contacts re-detected at every ALM iterate, stateful drive velocities and
per-step joint reference orientations.  An implicit-function adjoint of the
final Newton solve alone would leave all of those out; differencing whole
rollouts keeps them, and the perturbed copies are independent worlds, which
is the work the batched launch is built for (2P + 1 worlds per Jacobian for P
parameters).

Parameters (ParamSpec.kinds, in this order in the flat vector):
  "velocity"        initial linear velocity of the chosen bodies  (3 each)
  "mass"            RigidBody::mass of the chosen bodies            (1 each)
  "friction"        the solver's friction coefficient               (1)
  "joint_stiffness" ALM penalty of the chosen joints                (1 each)
Outputs: final position (3) and orientation (w, x, y, z) of the chosen
bodies, flattened.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Sequence

import numpy as np

from . import abi
from .scenes import Scene


@dataclasses.dataclass
class ParamSpec:
    kinds: Sequence[str]
    bodies: Sequence[int] = ()          # world indices for velocity / mass
    joints: Sequence[int] = ()          # joint indices for joint_stiffness

    def size(self) -> int:
        n = 0
        for k in self.kinds:
            n += {"velocity": 3 * len(self.bodies), "mass": len(self.bodies), "friction": 1,
                  "joint_stiffness": len(self.joints)}[k]
        return n

    def get(self, sc: Scene) -> np.ndarray:
        out = []
        for k in self.kinds:
            if k == "velocity":
                out.extend(sc.velocity[list(self.bodies)].reshape(-1))
            elif k == "mass":
                out.extend(sc.mass[list(self.bodies)])
            elif k == "friction":
                out.append(sc.settings.friction_coeff)
            elif k == "joint_stiffness":
                out.extend(sc.joint_stiffness[list(self.joints)])
            else:
                raise ValueError(f"unknown parameter kind {k!r}")
        return np.asarray(out, dtype=np.float64)

    def put(self, sc: Scene, theta) -> Scene:
        """A copy of sc with the parameters set to theta."""
        theta = np.asarray(theta, dtype=np.float64)
        s = abi.NxdSettings.from_buffer_copy(sc.settings)
        new = dataclasses.replace(sc, velocity=sc.velocity.copy(), mass=sc.mass.copy(),
                                  joint_stiffness=sc.joint_stiffness.copy(), settings=s)
        o = 0
        for k in self.kinds:
            if k == "velocity":
                n = 3 * len(self.bodies)
                new.velocity[list(self.bodies)] = theta[o:o + n].reshape(-1, 3)
            elif k == "mass":
                n = len(self.bodies)
                new.mass[list(self.bodies)] = theta[o:o + n]
            elif k == "friction":
                n = 1
                new.settings.friction_coeff = float(theta[o])
            else:
                n = len(self.joints)
                new.joint_stiffness[list(self.joints)] = theta[o:o + n]
            o += n
        return new


def final_poses(state: dict, bodies: Sequence[int]) -> np.ndarray:
    b = list(bodies)
    return np.concatenate([state["position"][b], state["orientation"][b]], axis=1).reshape(-1)


def batch_runner(scenes: Sequence[Scene], steps: int) -> list:
    """Step every scene `steps` times as one device batch; final states."""
    from .runtime import Batch
    b = Batch(scenes)
    try:
        b.step(steps)
        return [b.state(i) for i in range(len(scenes))]
    finally:
        b.close()


Runner = Callable[[Sequence[Scene], int], list]


def rollout(scene: Scene, spec: ParamSpec, theta, steps: int, out_bodies: Sequence[int],
            runner: Runner = batch_runner) -> np.ndarray:
    """Final poses of out_bodies after `steps` steps with parameters theta."""
    return final_poses(runner([spec.put(scene, theta)], steps)[0], out_bodies)


def rollout_jacobian(scene: Scene, spec: ParamSpec, theta, steps: int, out_bodies: Sequence[int],
                     h: float | np.ndarray = 1e-6, runner: Runner = batch_runner):
    """(y, J): final poses y(theta) of out_bodies after `steps` steps and
    J = dy/dtheta by central differences with step h (relative to
    max(1, |theta_i|) when h is a scalar), all 2P + 1 rollouts in one batch."""
    theta = np.asarray(theta, dtype=np.float64)
    P = theta.size
    hv = np.broadcast_to(np.asarray(h, dtype=np.float64), (P,)) * (np.maximum(1.0, np.abs(theta))
                                                                  if np.ndim(h) == 0 else 1.0)
    worlds = [spec.put(scene, theta)]
    for i in range(P):
        for sgn in (1.0, -1.0):
            t = theta.copy()
            t[i] += sgn * hv[i]
            worlds.append(spec.put(scene, t))
    states = runner(worlds, steps)
    y = final_poses(states[0], out_bodies)
    J = np.empty((y.size, P))
    for i in range(P):
        yp = final_poses(states[1 + 2 * i], out_bodies)
        ym = final_poses(states[2 + 2 * i], out_bodies)
        J[:, i] = (yp - ym) / (2.0 * hv[i])
    return y, J


def rollout_function(scene: Scene, spec: ParamSpec, steps: int, out_bodies: Sequence[int], h=1e-6,
                     runner: Runner = batch_runner):
    """A torch.autograd.Function: theta (float64 tensor) -> final poses, whose
    backward multiplies by the batched central-difference Jacobian."""
    import torch

    class Rollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta):
            y, J = rollout_jacobian(scene, spec, theta.detach().cpu().numpy(), steps, out_bodies, h, runner)
            ctx.save_for_backward(torch.from_numpy(J).to(theta.device))
            return torch.from_numpy(y).to(theta.device)

        @staticmethod
        def backward(ctx, grad_y):
            (J,) = ctx.saved_tensors
            return J.t() @ grad_y

    return Rollout.apply


def fit(scene: Scene, spec: ParamSpec, theta0, target, steps: int, out_bodies: Sequence[int], iters: int = 5,
        h=1e-6, damping: float = 1e-9, runner: Runner = batch_runner):
    """Parameter identification: damped Gauss-Newton on |y(theta) - target|^2
    with the batched Jacobian.  Returns (theta, loss history)."""
    theta = np.asarray(theta0, dtype=np.float64).copy()
    hist = []
    for _ in range(iters):
        y, J = rollout_jacobian(scene, spec, theta, steps, out_bodies, h, runner)
        r = y - np.asarray(target, dtype=np.float64)
        hist.append(float(r @ r))
        A = J.T @ J + damping * np.eye(theta.size)
        theta = theta - np.linalg.solve(A, J.T @ r)
    r = rollout(scene, spec, theta, steps, out_bodies, runner) - np.asarray(target, dtype=np.float64)
    hist.append(float(r @ r))
    return theta, hist
