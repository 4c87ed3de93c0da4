"""Independent scenes sharded over the ranks of a job, one GPU per rank.

Scenes of a batch never interact, so a batch splits across GPUs with no
exchange while it steps: each rank builds an `nxd_batch` of its share and
steps it on its own device; at the end the per-scene results are gathered.
The reference steps each scene on its own (`IPCSolver::step`, one World per
scene, IPCSolver.cpp:808); a batch of scenes has no counterpart there.

Assignment is greedy longest-processing-time: scenes in descending order of
estimated cost, each to the rank with the least total so far (ties to the
lower rank), which keeps the slowest rank within one scene's cost of the
mean.  The cost estimate is the per-step work that grows with a scene: its
bodies (pose, inertia, Newton DOFs), its joints and control forms (Newton
items) and its mesh primitives (broad and narrow phase).
"""
from __future__ import annotations

import numpy as np


def scene_cost(scene) -> float:
    """Estimated relative cost of one step of `scene`."""
    n = scene.n_bodies
    joints = int(scene.joint_type.shape[0])
    drives = int(scene.drive_body_b.shape[0])
    return 6.0 * n + 12.0 * joints + 4.0 * drives + 0.05 * (scene.n_faces + scene.n_vertices)


def assign(costs, world_size: int):
    """Per rank, the ascending scene indices it steps (greedy LPT)."""
    costs = np.asarray(costs, dtype=np.float64)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = np.zeros(world_size)
    parts = [[] for _ in range(world_size)]
    for i in order:
        r = int(np.argmin(load))            # first minimum: the lowest rank on ties
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def my_scenes(scenes, rank: int, world_size: int):
    """(indices, scenes) of this rank's share."""
    idx = assign([scene_cost(s) for s in scenes], world_size)[rank]
    return idx, [scenes[i] for i in idx]


def gather(results: dict, n_scenes: int):
    """All ranks' {scene index: result} merged into a list ordered by scene
    index (every rank receives it).  One all_gather of Python objects over the
    job's process group, after stepping; without a group of more than one
    rank the local results are the whole list."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, results)
    else:
        parts = [results]
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"scene {k} was stepped by more than one rank")
            merged[k] = v
    missing = [i for i in range(n_scenes) if i not in merged]
    if missing:
        raise RuntimeError(f"scenes {missing[:8]} were stepped by no rank")
    return [merged[i] for i in range(n_scenes)]


def step_sharded(scenes, steps: int, rank: int, world_size: int):
    """Steps this rank's share of `scenes` as one batch on the current GPU,
    `steps` steps, and returns every scene's final state and diagnostics in
    scene order (gathered from all ranks)."""
    from . import runtime
    idx, mine = my_scenes(scenes, rank, world_size)
    out = {}
    if mine:
        b = runtime.Batch(mine)
        b.step(steps)
        for k, i in enumerate(idx):
            out[i] = {"state": b.state(k), "diagnostics": b.diagnostics(k)}
        b.close()
    return gather(out, len(scenes))
