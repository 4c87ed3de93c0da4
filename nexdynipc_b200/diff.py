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
  "inertia"         body-frame inertia diagonal entries
                    ParamSpec.inertia_axes of the chosen bodies     (1 per axis)
  "friction"        the solver's friction coefficient               (1)
  "joint_stiffness" ALM penalty of the chosen joints                (1 each)
Outputs: final position (3) and orientation (w, x, y, z) of the chosen
bodies, flattened (rollout_jacobian), or their positions sampled along the
rollout (trajectory_jacobian).

Identification against measured trajectories follows the reference's
comparison workflow (tools/compare_with_reference.py): trajectory files of
time and x, y, z columns under one header row (load_reference_csv), the
reference interpolated at the simulation's sample times (reference_at), and
the RMSE of the Euclidean distance between the two (rmse_distance);
fit_trajectory runs Gauss-Newton on that residual.
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
    bodies: Sequence[int] = ()          # world indices for velocity / mass / inertia
    joints: Sequence[int] = ()          # joint indices for joint_stiffness
    inertia_axes: Sequence[int] = (0, 1, 2)   # diagonal entries for "inertia"

    def _count(self, k: str) -> int:
        n = {"velocity": 3 * len(self.bodies), "mass": len(self.bodies),
             "inertia": len(self.bodies) * len(self.inertia_axes), "friction": 1,
             "joint_stiffness": len(self.joints)}.get(k)
        if n is None:
            raise ValueError(f"unknown parameter kind {k!r}")
        return n

    def size(self) -> int:
        return sum(self._count(k) for k in self.kinds)

    def feasible(self, theta) -> bool:
        """Masses, inertias and joint stiffnesses positive, friction >= 0."""
        theta = np.asarray(theta, dtype=np.float64)
        if not np.all(np.isfinite(theta)):
            return False
        o = 0
        for k in self.kinds:
            n = self._count(k)
            seg = theta[o:o + n]
            if (k in ("mass", "inertia", "joint_stiffness") and np.any(seg <= 0.0)) or (k == "friction" and np.any(seg < 0.0)):
                return False
            o += n
        return True

    def get(self, sc: Scene) -> np.ndarray:
        out = []
        for k in self.kinds:
            if k == "velocity":
                out.extend(sc.velocity[list(self.bodies)].reshape(-1))
            elif k == "mass":
                out.extend(sc.mass[list(self.bodies)])
            elif k == "inertia":
                out.extend(sc.inertia[b, 4 * a] for b in self.bodies for a in self.inertia_axes)
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
        new = dataclasses.replace(sc, velocity=sc.velocity.copy(), mass=sc.mass.copy(), inertia=sc.inertia.copy(),
                                  joint_stiffness=sc.joint_stiffness.copy(), settings=s)
        o = 0
        for k in self.kinds:
            n = self._count(k)
            if k == "velocity":
                new.velocity[list(self.bodies)] = theta[o:o + n].reshape(-1, 3)
            elif k == "mass":
                new.mass[list(self.bodies)] = theta[o:o + n]
            elif k == "inertia":
                i = o
                for b in self.bodies:
                    for a in self.inertia_axes:
                        new.inertia[b, 4 * a] = theta[i]
                        i += 1
            elif k == "friction":
                new.settings.friction_coeff = float(theta[o])
            else:
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


def _perturbed(scene: Scene, spec: ParamSpec, theta, h):
    """The 2P + 1 worlds of a central-difference Jacobian (theta, then
    theta +- h_i e_i for each i) and the steps h_i (relative to
    max(1, |theta_i|) when h is a scalar)."""
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
    return worlds, hv


def _central(outputs: list, hv: np.ndarray):
    """(y, J) from the outputs of _perturbed's worlds."""
    y = outputs[0]
    J = np.empty((y.size, hv.size))
    for i in range(hv.size):
        J[:, i] = (outputs[1 + 2 * i] - outputs[2 + 2 * i]) / (2.0 * hv[i])
    return y, J


def rollout_jacobian(scene: Scene, spec: ParamSpec, theta, steps: int, out_bodies: Sequence[int],
                     h: float | np.ndarray = 1e-6, runner: Runner = batch_runner):
    """(y, J): final poses y(theta) of out_bodies after `steps` steps and
    J = dy/dtheta by central differences with step h (relative to
    max(1, |theta_i|) when h is a scalar), all 2P + 1 rollouts in one batch."""
    worlds, hv = _perturbed(scene, spec, theta, h)
    states = runner(worlds, steps)
    return _central([final_poses(st, out_bodies) for st in states], hv)


def sample_counts(steps: int, every: int) -> np.ndarray:
    """Step counts at which a sampled rollout records states: every, 2 every,
    ..., and `steps` itself when it is not a multiple of every."""
    if steps < 1 or every < 1:
        raise ValueError("steps and every must be positive")
    c = list(range(every, steps + 1, every))
    if c[-1:] != [steps]:
        c.append(steps)
    return np.asarray(c)


def batch_sampler(scenes: Sequence[Scene], steps: int, every: int) -> list:
    """Step every scene `steps` times as one device batch; per scene, its
    states at sample_counts(steps, every)."""
    from .runtime import Batch
    b = Batch(scenes)
    try:
        out = [[] for _ in scenes]
        done = 0
        for c in sample_counts(steps, every):
            b.step(int(c) - done)
            done = int(c)
            for i in range(len(scenes)):
                out[i].append(b.state(i))
        return out
    finally:
        b.close()


Sampler = Callable[[Sequence[Scene], int, int], list]


def sampled_positions(states: list, bodies: Sequence[int]) -> np.ndarray:
    """Positions of `bodies` at each sampled state, flattened sample-major."""
    b = list(bodies)
    return np.concatenate([st["position"][b].reshape(-1) for st in states])


def trajectory_jacobian(scene: Scene, spec: ParamSpec, theta, steps: int, out_bodies: Sequence[int], every: int,
                        h: float | np.ndarray = 1e-6, sampler: Sampler = batch_sampler):
    """(t, y, J): sample times t = dt * sample_counts(steps, every), the
    positions y(theta) of out_bodies at those times (sample-major, then body,
    then x, y, z) and J = dy/dtheta by central differences, all 2P + 1
    rollouts stepped as one batch."""
    worlds, hv = _perturbed(scene, spec, theta, h)
    runs = sampler(worlds, steps, every)
    y, J = _central([sampled_positions(r, out_bodies) for r in runs], hv)
    return scene.dt * sample_counts(steps, every), y, J


def load_reference_csv(path: str) -> np.ndarray:
    """(n, 4) float64 rows of time, x, y, z from a reference trajectory file
    (nexdynipc/assets/reference_data/<case>/<Body>_<Pos|Vel|Acc>.csv: one
    header row, time in column 0 and the three components in columns 1-3,
    the columns tools/compare_with_reference.py:37-80 reads)."""
    return np.loadtxt(path, delimiter=",", skiprows=1, usecols=(0, 1, 2, 3), ndmin=2)


def reference_at(t, ref: np.ndarray) -> np.ndarray:
    """The reference trajectory linearly interpolated at times t, (len(t), 3)
    (compare_with_reference.py:120-126: np.interp per component)."""
    t = np.asarray(t, dtype=np.float64)
    return np.stack([np.interp(t, ref[:, 0], ref[:, i]) for i in (1, 2, 3)], axis=1)


def rmse_distance(sim, ref) -> float:
    """sqrt(mean_i |sim_i - ref_i|^2) over (n, 3) samples
    (compare_with_reference.py:82-83,129-136)."""
    d = np.linalg.norm(np.asarray(sim, dtype=np.float64) - np.asarray(ref, dtype=np.float64), axis=1)
    return float(np.sqrt(np.mean(d ** 2)))


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


def fit_trajectory(scene: Scene, spec: ParamSpec, theta0, target, steps: int, out_bodies: Sequence[int], every: int,
                   iters: int = 6, h=1e-6, damping: float = 1e-9, sampler: Sampler = batch_sampler,
                   max_halvings: int = 8):
    """Parameter identification on a sampled trajectory: Gauss-Newton on
    |y(theta) - target|^2 with y and its Jacobian from trajectory_jacobian
    (target laid out like y), each step halved until it is feasible
    (ParamSpec.feasible) and lowers the loss, at most max_halvings times;
    stops early when no halving lowers it.  Returns (theta, loss history)."""
    theta = np.asarray(theta0, dtype=np.float64).copy()
    target = np.asarray(target, dtype=np.float64)
    hist = []
    for _ in range(iters):
        _, y, J = trajectory_jacobian(scene, spec, theta, steps, out_bodies, every, h, sampler)
        r = y - target
        loss = float(r @ r)
        hist.append(loss)
        step = -np.linalg.solve(J.T @ J + damping * np.eye(theta.size), J.T @ r)
        accepted = False
        for _ in range(max_halvings + 1):
            trial = theta + step
            if spec.feasible(trial):
                yt = sampled_positions(sampler([spec.put(scene, trial)], steps, every)[0], out_bodies)
                if float((yt - target) @ (yt - target)) < loss:
                    theta, accepted = trial, True
                    break
            step = 0.5 * step
        if not accepted:
            return theta, hist
    yt = sampled_positions(sampler([spec.put(scene, theta)], steps, every)[0], out_bodies)
    hist.append(float((yt - target) @ (yt - target)))
    return theta, hist


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
