#!/usr/bin/env python3
"""Benchmark of the B200 contact step (IPCSolver::step of NexDynIPC).

Workload: the 1024-body hopper scene (1024 convex hulls of 64 seeded sphere
points scaled to 0.05 m in a 1x1x4 m open hopper, plus 32 hinge chains of 8
links with angle limits; 1313 bodies; dt 5e-3, dhat 5e-4, mu 0.3, 2 ALM
iterations), generated from a seed (no dataset).  A step is one
IPCSolver::step.  Prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank steps its own replica of the scene on its GPU (the
single-scene step does not shard: replicas only); the value is the steps of
all ranks divided by the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s @1024 bodies (1e-6 traj err), GPU plain vs batched; fwd+adj/fwd time"
UNIT = "steps/s"
WORKLOAD = ("hopper_chains: 1024 convex hulls (64 seeded sphere points, 124 tris, scaled 0.05 m) in a 1x1x4 m "
            "open hopper + 32 hinge chains x 8 links with +-60 deg angle limits; 1313 bodies, 130442 tris; "
            "dt=5e-3, dhat=5e-4, mu=0.3, 2 ALM iterations; FP64")
FAMILIES = ["assembly", "broad_phase", "topk", "narrow_phase", "min_distance", "newton", "alm_post", "scan", "other"]


def max_over_ranks(x: float, device: str = "cuda") -> float:
    """The largest x over the ranks of the process group (the timing rule for
    several GPUs: the job takes as long as its slowest rank); x itself when
    no group of more than one rank is running."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                vals = [v.strip() for v in out.stdout.strip().split(",")]
                if len(vals) >= 7:
                    self.samples.append(vals)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def candidate_operand_bytes(fv: int, ee: int, contacts: int) -> int:
    """Operand bytes of one narrow-phase pass counted per candidate: per
    face-vertex candidate 16 B of ids + 4 x 24 B of vertex coordinates, per
    edge-edge candidate 24 B + 4 x 24 B; 88 B per contact written."""
    return fv * (16 + 96) + ee * (24 + 96) + contacts * 88


def staged_pair_bytes(n_pairs: int, contacts: int) -> int:
    """Bytes one narrow-phase pass must move: per body pair its two ids, the
    six top-32 id lists (768 B + 24 B of sizes), the coordinates of the 64
    selected vertices (24 B each), the 64 selected faces (12 B of ids + 3 x
    24 B of coordinates) and the 64 selected edges (8 B + 2 x 24 B), each
    read once per pair; 88 B per contact written."""
    return n_pairs * (8 + 768 + 24 + 64 * 24 + 64 * 84 + 64 * 56) + contacts * 88


def ncu_traffic():
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    from the ncu summaries under profiles/ ('traffic <kernel> <bytes>')."""
    out = {}
    pdir = os.path.join(ROOT, "profiles")
    for fn in sorted(os.listdir(pdir)) if os.path.isdir(pdir) else []:
        with open(os.path.join(pdir, fn)) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 3 and parts[0] == "traffic":
                    out[parts[1]] = int(parts[2])
    return out


def newton_bytes(n_bodies: int, n_joints: int, n_contacts: float) -> float:
    """Compulsory bytes of one Newton iteration of the block-sparse direct
    solve: every 6x6 Hessian block (bodies, joint and contact couplings)
    written and read once (2 x 288 B), seven passes over 6N-vectors (x, g,
    contact gradient, dx, trial x: 8 B x 6N each), 88 B per contact and about
    800 B of parameters, multipliers and Jacobian per joint."""
    return 2 * 288.0 * (n_bodies + n_joints + n_contacts) + 7 * 48.0 * n_bodies + 88.0 * n_contacts + 800.0 * n_joints


def oracle_steps(scene_fn, threads: int, skip: int, steps: int, literal: bool):
    """The CPU oracle (the reference's step restated) on the same scene and
    step indices as the device: `skip` untimed steps with the pruned scene
    minimum distance (exact below 1e-6, so its stiffness decisions and the
    trajectory are the literal loop's), then `steps` steps timed one by one
    (wall clock) with the literal O(N^2 V F) loop of
    AdaptiveBarrier::computeSceneMinDistance (literal=True) or the pruned one.
    Returns (seconds per timed step, untimed seconds)."""
    from oracle.refcpu import OracleWorld
    sc = scene_fn()
    ow = OracleWorld(sc, literal_min_distance=False, threads=threads)
    t0 = time.perf_counter()
    for _ in range(skip):
        ow.step()
    ff = time.perf_counter() - t0
    ow.set_options(literal_min_distance=literal, threads=threads)
    walls = []
    for _ in range(steps):
        t1 = time.perf_counter()
        ow.step()
        walls.append(time.perf_counter() - t1)
    ow.close()
    return walls, ff


def batched_leg(torch, steps: int, warmup: int, flush, ws: int = 1, rank: int = 0, plain: bool = True):
    """256 independent scenes of 2-63 bodies (the batched configuration, seed
    4000): aggregate scene-steps/s of the batched form (one graph of batched
    launches per step) next to the plain path (the same scenes, one context
    each, stepped one after another on one stream).  Both device-timed with
    CUDA events per step, L2 flushed between steps.  Under several ranks the
    scenes are sharded (nexdynipc_b200.shard: greedy by estimated cost, no
    exchange while stepping): each rank steps its share, the time is the
    slowest rank's, the value all 256 scenes' steps over it."""
    from nexdynipc_b200 import runtime, scenes, shard
    all_scs = scenes.batched_scenes(n_scenes=256)
    idx, scs = shard.my_scenes(all_scs, rank, ws)
    stream = torch.cuda.Stream()
    lib = runtime.lib()
    # the queue grids of the narrow phase, tuned on a throwaway batch of the
    # same scenes (the tuning steps it), then applied to the timed one
    import tempfile
    tb = runtime.Batch(scs)
    with tempfile.TemporaryDirectory() as td:
        tune = tb.autotune(cache_path=os.path.join(td, "autotune.json"), steps=2)
    tb.close()
    b = runtime.Batch(scs)
    for kname, v in tune["choice"].items():
        b.set_queue_ctas(runtime.QUEUE_KERNELS[kname], v)
    b.set_stream(stream.cuda_stream)
    singles = [runtime.Context(s) for s in scs] if plain else []
    for c in singles:
        lib.nxd_set_stream(c.h, C.c_void_p(stream.cuda_stream))

    def plain_step():
        for c, s in zip(singles, scs):
            st = lib.nxd_step(c.h, s.dt)
            if st != 0:
                raise runtime.NxdError("nxd_step", st)

    def timed(fn):
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.fill_(k & 0xFF)
                ev[k][0].record(stream)
                fn()
                ev[k][1].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(e) for a, e in ev) / 1e3

    if ws > 1:
        torch.distributed.barrier()
    t_batched = max_over_ranks(timed(b.step))
    t_plain = max_over_ranks(timed(plain_step)) if plain else None
    status = max(b.diagnostics(i)["status"] for i in range(len(scs)))
    same = plain and all(np.array_equal(b.state(i)["position"], singles[i].state()["position"])
                         for i in range(0, len(scs), 17))
    n = len(all_scs)
    out = {"scenes": n, "bodies": int(sum(s.n_bodies for s in all_scs)), "steps": steps,
           "value": n * steps / t_batched, "plain_value": n * steps / t_plain if plain else None, "unit": "scene-steps/s",
           "batched_over_plain": t_plain / t_batched if plain else None, "groups": b.groups(), "status": int(status),
           "equal_to_plain_sample": bool(same), "ranks": ws, "scenes_this_rank": len(scs),
           "queue_ctas_per_sm": tune["choice"], "autotune_ms": {k: round(v, 3) for k, v in tune["timings_ms"].items()},
           "sharding": "greedy by estimated cost, no exchange while stepping" if ws > 1 else "one rank"}
    for c in singles:
        c.close()
    b.close()
    return out


def full_run_leg(torch, lib, stream, flush):
    """The workload's whole run: a fresh context of the same scene stepped
    through all its steps (100), each step its CUDA graph, CUDA events per
    step, L2 flushed between steps.  The bench's K-step window sits early in
    the run; the pile forms later, so this is the configuration's full cost."""
    from nexdynipc_b200 import runtime, scenes
    sc = scenes.hopper_chains()
    ctx = runtime.Context(sc)
    lib.nxd_set_stream(ctx.h, C.c_void_p(stream.cuda_stream))
    n = sc.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(n):
            flush.fill_(k & 0xFF)
            ev[k][0].record(stream)
            st = lib.nxd_step(ctx.h, sc.dt)
            if st != 0:
                raise runtime.NxdError("nxd_step", st)
            ev[k][1].record(stream)
    torch.cuda.synchronize()
    ms = np.array([a.elapsed_time(b) for a, b in ev])
    d = ctx.diagnostics()
    ctx.close()
    return {"steps": n, "steps_per_s": n / (ms.sum() / 1e3), "ms_total": float(ms.sum()),
            "steps_per_s_1_50": 50 / (ms[:50].sum() / 1e3), "steps_per_s_51_100": 50 / (ms[50:].sum() / 1e3),
            "ms_max_step": float(ms.max()), "slowest_step": int(np.argmax(ms)) + 1, "status": int(d["status"])}


def diff_leg(torch):
    """Differentiable-rollout configuration: 16 icospheres colliding on a
    ground box, 50 steps, final poses differentiated with respect to the 48
    initial velocities, 16 masses and the friction coefficient by central
    differences, i.e. 131 worlds stepped as one batch.  Reports the device
    time of the 50 batched steps (CUDA events) and the wall time of the whole
    Jacobian call (scene copies, batch creation, read-back), and the ratio
    of the Jacobian's device time to one forward rollout's (forward plus
    gradient over forward)."""
    import time
    from nexdynipc_b200 import diff, runtime, scenes
    sc = scenes.diff_scene()
    bodies = list(range(1, sc.n_bodies))
    spec = diff.ParamSpec(["velocity", "mass", "friction"], bodies=bodies)
    theta = spec.get(sc)
    steps = sc.steps
    times = {}

    def runner(worlds, n):
        stream = torch.cuda.Stream()
        b = runtime.Batch(worlds)
        b.set_stream(stream.cuda_stream)
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            a.record(stream)
            b.step(n)
            e.record(stream)
        torch.cuda.synchronize()
        times["device_s"] = a.elapsed_time(e) / 1e3
        out = [b.state(i) for i in range(len(worlds))]
        status = max(b.diagnostics(i)["status"] for i in range(len(worlds)))
        b.close()
        times["status"] = status
        return out

    diff.rollout_jacobian(sc, spec, theta, 2, bodies, runner=runner)      # warm-up (module load, graphs)
    runner([sc], steps)                                                   # the forward rollout alone
    fwd_s = times["device_s"]
    t0 = time.perf_counter()
    y, J = diff.rollout_jacobian(sc, spec, theta, steps, bodies, runner=runner)
    wall = time.perf_counter() - t0
    worlds = 2 * theta.size + 1
    return {"workload": f"{sc.n_bodies - 1} icospheres (162 V) on a ground box, {steps} steps, dt {sc.dt}",
            "parameters": int(theta.size), "outputs": int(y.size), "worlds": worlds,
            "device_s": times["device_s"], "wall_s": wall, "forward_device_s": fwd_s,
            "fwd_plus_grad_over_fwd": times["device_s"] / fwd_s,
            "scene_steps_per_s": worlds * steps / times["device_s"],
            "jacobians_per_s_wall": 1.0 / wall, "status": int(times["status"]),
            "finite": bool(np.isfinite(J).all())}


def adjoint_leg(torch, n_sets: int = 2):
    """Differentiable configuration on the full-IPC step: 16 icospheres
    (162 V) over a ground box, 50 steps, loss = squared error of the final
    poses against a seeded target, gradients with respect to every initial
    velocity, mass, the ground joint's stiffness and the friction coefficient
    by the adjoint (nxd_ipc_adjoint per step, checkpoints every 10 steps, each
    segment re-stepped in the backward pass), through torch.autograd.  The
    step has lagged friction (mu 0.4, eps 1e-5 m, one lagging pass).  Wall
    clock of the forward rollout and of the backward pass, per parameter set
    (the initial velocities perturbed per set), the sets one after another."""
    from nexdynipc_b200 import abi, adjoint, runtime, scenes
    params = abi.ipc_params(dhat=1e-3, kappa=1e9, eta=0.1, newton_tol=1e-9, newton_max_iters=100, ls_max_iters=40,
                            mu=0.4, friction_eps=1e-5, friction_iters=1)
    base = scenes.diff_ipc_scene()
    fn = adjoint.make_rollout_function()
    rng = np.random.default_rng(5100)
    fwd, bwd, gnorm, gfric = [], [], [], []
    for k in range(n_sets):
        v0 = torch.tensor(base.velocity + rng.normal(0, 0.05, base.velocity.shape), requires_grad=True)
        m = torch.tensor(base.mass, requires_grad=True)
        mu = torch.tensor(base.joint_stiffness, requires_grad=True)
        fr = torch.tensor(0.4, dtype=torch.float64, requires_grad=True)
        tgt = torch.tensor(np.concatenate([base.position, base.orientation], 1) + rng.normal(0, 0.02, (base.n_bodies, 7)))
        t0 = time.perf_counter()
        out = fn.apply(v0, m, mu, base, params, base.steps, 10, fr)
        t1 = time.perf_counter()
        loss = ((out - tgt) ** 2).sum()
        loss.backward()
        t2 = time.perf_counter()
        fwd.append(t1 - t0)
        bwd.append(t2 - t1)
        gnorm.append(float(v0.grad.abs().max()))
        gfric.append(float(fr.grad))
    return {"workload": (f"{base.n_bodies - 1} icospheres (162 V) on a ground box (fixed joint 1e5), {base.steps} "
                         f"steps, dt {base.dt}, full-IPC step (kappa 1e9, dhat 1e-3, Newton |g| < 1e-9), lagged "
                         f"friction mu 0.4"),
            "parameter_sets": n_sets, "parameters_per_set": int(3 * base.n_bodies + base.n_bodies + 1 + 1),
            "checkpoint_every": 10, "forward_s": float(np.mean(fwd)), "backward_s": float(np.mean(bwd)),
            "fwd_plus_adj_over_fwd": float(np.mean([(a + b) / a for a, b in zip(fwd, bwd)])),
            "max_abs_velocity_gradient": gnorm, "friction_coefficient_gradient": gfric,
            "timing": "wall clock; the backward pass re-steps each 10-step segment from its checkpoint"}


def pcg_leg(n_bodies: int = 200000, iters: int = 60):
    """Block-Jacobi PCG (nxd_pcg_solve) on a synthetic SPD block system of
    the size a large full-IPC Newton system reaches: n_bodies 6x6 block rows,
    each coupled to its neighbours at offsets 1, 64 and 4096 (7 blocks per
    row, 400 MB of blocks at 200k bodies, far above L2), tol 0 so that
    exactly `iters` iterations run; CUDA-event time of the iteration kernel.
    The iteration reads the upper block triangle.  Algorithmic bytes per
    iteration: each stored off-diagonal block once (288 B + 4 B column), the
    diagonal and inverse diagonal blocks as 21 doubles each, the row
    pointers of both triangles, the lower entries' block index and row (8 B
    each), thirteen 6N-vector passes."""
    from nexdynipc_b200 import runtime, scenes
    rng = np.random.default_rng(9000)
    n = n_bodies
    rows, cols, blks = [np.arange(n)], [np.arange(n)], []
    M = rng.normal(size=(n, 6, 6)) * 0.05
    blks.append(np.einsum("nij,nkj->nik", M, M) + (1.0 + 36 * 0.1) * np.eye(6))
    for o in (1, 64, 4096):
        i = np.arange(n - o)
        B = rng.uniform(-0.1, 0.1, size=(n - o, 6, 6))
        rows += [i, i + o]
        cols += [i + o, i]
        blks += [B, np.transpose(B, (0, 2, 1))]
    r, c = np.concatenate(rows), np.concatenate(cols)
    order = np.lexsort((c, r))
    ci = np.ascontiguousarray(c[order], dtype=np.int32)
    vals = np.ascontiguousarray(np.concatenate(blks)[order].reshape(-1, 36))
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    rp = np.cumsum(rp).astype(np.int32)
    b = rng.normal(size=6 * n)
    sb = scenes.SceneBuilder("host")
    sb.add_body(np.zeros((0, 3)), np.zeros((0, 3), np.int32), (0.0, 0.0, 0.0), mass=1.0, inertia=np.eye(3))
    from nexdynipc_b200 import abi
    ctx = runtime.Context(sb.build(abi.default_settings(), 0.01, 1))
    ctx.pcg_solve(rp, ci, vals, b, tol=0.0, max_iter=3, check=False)           # warm-up
    x, st = ctx.pcg_solve(rp, ci, vals, b, tol=0.0, max_iter=iters, check=False)
    ctx.close()
    nnzb = len(ci)
    n_up = (nnzb - n) // 2
    per_iter = 292.0 * n_up + 8.0 * n_up + 8.0 * (n + 1) + 2 * 168.0 * n + 13 * 48.0 * n
    secs = st["kernel_ms"] / 1e3
    return {"bodies": n, "blocks": nnzb, "stored_blocks": n_up, "iterations": st["iterations"], "kernel_ms": st["kernel_ms"],
            "ms_per_iteration": st["kernel_ms"] / max(st["iterations"], 1), "relative_residual": st["relative_residual"],
            "grid": st["grid"], "threads": st["threads"], "bytes_per_iteration": per_iter,
            "achieved_gbs": per_iter * st["iterations"] / secs / 1e9 if secs > 0 else None}


def ipc_step_params(solver: int = 0, mu: float = 0.0):
    from nexdynipc_b200 import abi, scenes
    return abi.ipc_params(**scenes.ipc_step_settings(solver, mu))


def ipc_step_leg(n_cubes: int = 8, columns: int = 1, settle: int = 30, steps: int = 20, solver: int = 0,
                 bowl: bool = False, mu: float = 0.0):
    """Full-IPC time step (nxd_ipc_step): after `settle` untimed steps, wall
    clock of `steps` steps, each a host-ordered Newton loop of device calls
    (candidates, barrier, rest forms, block solve, CCD bound, line search).
    The scene is stacks of tilted cubes falling onto a ground box, or with
    `bowl` the 64-sphere bowl configuration (642-vertex icospheres, 1280-face
    bowl); mu > 0 adds lagged friction.  One untimed step on a throwaway
    context of the same scene first loads the kernels; per-step wall times are
    kept so that a CPU sample of the first steps can be compared step for step."""
    import time
    from nexdynipc_b200 import runtime, scenes
    sc = scenes.sphere_bowl() if bowl else scenes.ipc_drop(n_cubes=n_cubes, columns=columns)
    p = ipc_step_params(solver, mu)
    warm = runtime.Context(sc)
    warm.ipc_step(p)
    warm.close()
    ctx = runtime.Context(sc)
    for _ in range(settle):
        ctx.ipc_step(p)
    its, act, pairs, conv, lsf, walls = [], [], [], 0, 0, []
    t0 = time.perf_counter()
    for _ in range(steps):
        t1 = time.perf_counter()
        st = ctx.ipc_step(p)
        walls.append(time.perf_counter() - t1)
        its.append(st["newton_iterations"]); act.append(st["n_active"]); pairs.append(st["n_pairs"])
        conv += st["converged"]
        lsf += st["line_search_failed"]
    wall = time.perf_counter() - t0
    ctx.close()
    fric = f", lagged friction mu {mu} (eps 1e-5 m, 2 passes)" if mu > 0 else ""
    if bowl:
        workload = (f"{sc.n_bodies - 1} icospheres (642 V) falling into a 1280-face bowl, full IPC, dhat 1e-3, "
                    f"kappa 1e11{fric}, dt {sc.dt}; steps {settle + 1}-{settle + steps}")
    else:
        workload = (f"{n_cubes} tilted 0.2 m cubes in {columns} stack(s) on a ground box, dhat 1e-3, "
                    f"kappa 1e11, dt {sc.dt}; steps {settle + 1}-{settle + steps}")
    return {"workload": workload,
            "steps": steps, "steps_per_s": steps / wall, "steps_per_s_median": 1.0 / float(np.median(walls)),
            "newton_iterations_mean": float(np.mean(its)),
            "active_pairs_mean": float(np.mean(act)), "candidate_pairs_mean": float(np.mean(pairs)),
            "converged_steps": conv, "line_search_failures": lsf, "friction_pairs_last": int(st["n_friction"]),
            "step_ms": [round(1e3 * w, 3) for w in walls[:4]],
            "linear_solver": "block-Jacobi PCG" if solver else "component LDL^T",
            "timing": "wall clock per nxd_ipc_step (it synchronises)"}


def ipc_step_cpu_baseline(n_cubes: int, columns: int, settle: int, steps: int, bowl: bool = False, mu: float = 0.0):
    """The CPU oracle's full-IPC step on the same trajectory segment as
    ipc_step_leg: `settle` untimed steps, then wall clock of `steps`.  The
    oracle's candidate search runs on all host threads (OpenMP), the rest of
    its step on one."""
    from nexdynipc_b200 import scenes
    from oracle.refcpu import OracleWorld
    ow = OracleWorld(scenes.sphere_bowl() if bowl else scenes.ipc_drop(n_cubes=n_cubes, columns=columns))
    p = ipc_step_params(0, mu)
    for _ in range(settle):
        ow.ipc_step(p)
    t0 = time.perf_counter()
    its, walls = 0, []
    for _ in range(steps):
        t1 = time.perf_counter()
        its += ow.ipc_step(p)["newton_iterations"]
        walls.append(time.perf_counter() - t1)
    wall = time.perf_counter() - t0
    return {"steps_per_s": steps / wall, "cores": os.cpu_count() or 1, "kind": "port", "newton_iterations_mean": its / steps,
            "step_ms": [round(1e3 * w, 1) for w in walls],
            "sample": (f"steps {settle + 1}-{settle + steps} through the CPU oracle's nxo_ipc_step (candidate search "
                       f"on all host threads, the rest serial), {wall:.2f} s wall")}


def mode_i_leg(ctx, sc, reps: int = 5):
    """Primitive-level contact model on the workload's current state, through
    the C ABI (host arrays in and out, each call synchronising): LBVH
    candidates (boxes inflated by dhat), the barrier form (energy, gradient,
    BSR Hessian) and the additive-CCD bound of the velocity step x -> x +
    dt v.  Median wall time of `reps` calls after one warm-up call."""
    st = ctx.state()
    n = sc.n_bodies
    x = np.zeros(6 * n)
    dx = np.zeros(6 * n)
    for i in range(n):
        x[6 * i:6 * i + 3] = st["position"][i]
        dx[6 * i:6 * i + 3] = sc.dt * st["velocity"][i]
        dx[6 * i + 3:6 * i + 6] = sc.dt * st["angular_velocity"][i]
    dhat, kappa = sc.settings.dhat, 1e6

    def timed(fn):
        fn()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            out = fn()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts)), out

    t_c, (pt, ee) = timed(lambda: ctx.ipc_candidates(x, None, dhat))
    t_b, (e, g, bsr, npairs, nact) = timed(lambda: ctx.ipc_barrier(x, dhat, kappa))
    t_s, (alpha, nccd) = timed(lambda: ctx.ipc_max_step(x, dx, 0.1))
    return {"candidates": {"ms": 1e3 * t_c, "pt_pairs": int(len(pt)), "ee_pairs": int(len(ee)),
                           "pairs_per_s": (len(pt) + len(ee)) / t_c},
            "barrier": {"ms": 1e3 * t_b, "pairs": int(npairs), "active": int(nact), "bsr_blocks": int(len(bsr[1])),
                        "pairs_per_s": npairs / t_b},
            "max_step": {"ms": 1e3 * t_s, "pairs": int(nccd), "alpha": alpha, "pairs_per_s": nccd / t_s},
            "timing": "wall clock per C-ABI call (host copies included), median of %d after a warm-up call" % reps,
            "primitives": {"vertices": int(sc.n_vertices), "faces": int(sc.n_faces)}}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args, ws, rank):
    """The reference arm: the reference's CPU step (the oracle's restatement:
    the reference itself cannot be built here) on the host's cores, over the
    step indices the device arm times.  The warm-up steps are fast-forwarded
    untimed with the pruned scene minimum distance (same trajectory), then
    each of the K timed steps runs the literal computeSceneMinDistance loop
    of the reference on all host threads.  A second, labelled leg times the
    first steps of the same window with the pruned loop (same trajectory,
    the GPU's pruning on the CPU), separating the algorithm from the
    hardware."""
    if rank != 0:
        return
    from nexdynipc_b200 import scenes
    threads = os.cpu_count() or 1
    walls, ff = oracle_steps(scenes.hopper_chains, threads, args.warmup, args.steps, literal=True)
    value = len(walls) / sum(walls)
    n_pruned = min(args.steps, 5)
    pwalls, pff = oracle_steps(scenes.hopper_chains, threads, args.warmup, n_pruned, literal=False)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(walls) / len(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "timed_steps": f"{args.warmup + 1}-{args.warmup + args.steps} (the device arm's window)",
                   "timed_s": sum(walls), "untimed_fast_forward_s": ff, "cpu": cpu_model(),
                   "pruned_steps_per_s": n_pruned / sum(pwalls),
                   "pruned_steps": f"{args.warmup + 1}-{args.warmup + n_pruned}"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": (f"steps {args.warmup + 1}-{args.warmup + args.steps} of the workload through the "
                                    f"CPU oracle (the reference's step restated; the reference cannot be built here: "
                                    f"Eigen/Boost absent) with {threads} OpenMP threads and the reference's literal "
                                    f"O(N^2 V F) computeSceneMinDistance, every step timed whole "
                                    f"({sum(walls):.1f} s); steps 1-{args.warmup} fast-forwarded untimed")},
        "cpu_baseline_pruned": {"value": n_pruned / sum(pwalls), "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": (f"steps {args.warmup + 1}-{args.warmup + n_pruned}, the same oracle with "
                                           f"the pruned scene minimum distance (identical trajectory), "
                                           f"{sum(pwalls):.1f} s")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-mode-i", action="store_true")
    ap.add_argument("--no-diff", action="store_true")
    ap.add_argument("--no-pcg", action="store_true")
    ap.add_argument("--adjoint-sets", type=int, default=2, help="parameter sets of the adjoint leg")
    ap.add_argument("--batched-only", type=int, metavar="STEPS",
                    help="only the batched form of the 256 scenes (1 warm-up step), one JSON line")
    ap.add_argument("--ipc-step-only", type=int, nargs=4, metavar=("CUBES", "COLUMNS", "SETTLE", "STEPS"),
                    help="run only the full-IPC step leg on that drop and print its JSON (for profiling)")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.ipc_step_only:
        n_cubes, columns, settle, steps = args.ipc_step_only
        print(json.dumps(ipc_step_leg(n_cubes=n_cubes, columns=columns, settle=settle, steps=steps)), flush=True)
        return
    if args.batched_only:
        import torch
        flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        print(json.dumps(batched_leg(torch, args.batched_only, 1, flush, plain=False)), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return

    import torch
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from nexdynipc_b200 import abi, runtime, scenes

    sc = scenes.hopper_chains()
    # three contexts of the same scene: the step is deterministic, so all pass
    # through identical states; ctx is timed (graph replay), ctx_prof steps
    # the same step indices with CUDA events around every launch, ctx_e2e
    # steps them again end to end through the C ABI with host buffers
    ctx = runtime.Context(sc)
    ctx_prof = runtime.Context(sc)
    ctx_e2e = runtime.Context(sc)
    lib = runtime.lib()
    stream = torch.cuda.Stream()
    for c_ in (ctx, ctx_prof, ctx_e2e):
        lib.nxd_set_stream(c_.h, C.c_void_p(stream.cuda_stream))
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")   # > 126 MB L2
    dt = sc.dt

    def step(c=ctx):
        st = lib.nxd_step(c.h, dt)
        if st != 0:
            raise runtime.NxdError("nxd_step", st)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
            step(ctx_prof)
            step(ctx_e2e)
    torch.cuda.synchronize()
    init_state = ctx.state()

    # --- device-timed steps (inputs resident in HBM), L2 flushed between
    # steps; each step is the context's captured CUDA graph (no per-launch
    # events inside the timed region)
    lib.nxd_profile(ctx.h, 0, None, None)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(k & 0xFF)
                starts[k].record(stream)
                step()
                ends[k].record(stream)
        torch.cuda.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    timed_n = np.zeros(9, dtype=np.int64)
    lib.nxd_profile(ctx.h, 0, None, timed_n.ctypes.data_as(C.POINTER(C.c_int64)))
    # --- the same step indices on the twin context with CUDA events around
    # every launch (direct launches): per-family device time
    prof_ms = np.zeros(9)
    prof_n = np.zeros(9, dtype=np.int64)
    lib.nxd_profile(ctx_prof.h, 1, None, None)
    prof_steps = []
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            step(ctx_prof)
            prof_steps.append(ctx_prof.diagnostics())   # synchronises; events bracket the launches only
    torch.cuda.synchronize()
    lib.nxd_profile(ctx_prof.h, 0, abi.dptr(prof_ms), prof_n.ctypes.data_as(C.POINTER(C.c_int64)))
    twin_equal = bool(np.array_equal(ctx.state()["position"], ctx_prof.state()["position"]))
    diag = ctx.diagnostics()
    total_ms = max_over_ranks(total_ms)
    value = ws * args.steps / (total_ms / 1e3)

    # --- narrow-phase item counts of the current candidate set (roofline units)
    cand_counts = ctx.candidate_counts(sc.settings.dhat) if hasattr(ctx, "candidate_counts") else None

    # --- end to end through the C ABI with pinned host buffers
    n = sc.n_bodies
    pinned = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in init_state.items()}
    out_pinned = {k: torch.empty_like(v).pin_memory() for k, v in pinned.items()}
    dp = C.POINTER(C.c_double)

    def view(d):
        return abi.NxdState(*[C.cast(C.c_void_p(d[k].data_ptr()), dp) for k in
                              ("position", "orientation", "velocity", "angular_velocity", "linear_acceleration",
                               "angular_acceleration")])

    vin, vout = view(pinned), view(out_pinned)
    h2d = sum(v.numel() * 8 for v in pinned.values())
    d2h = sum(v.numel() * 8 for v in out_pinned.values())
    # a host-driven loop over the same step indices as the device-timed
    # steps (ctx_e2e took the same warm-up steps): each step uploads the
    # state the previous step read back
    lib.nxd_get_state(ctx_e2e.h, C.byref(vin))
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lib.nxd_set_state(ctx_e2e.h, C.byref(vin))
        step(ctx_e2e)
        lib.nxd_get_state(ctx_e2e.h, C.byref(vout))
        vin, vout = vout, vin
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s)
    e2e = ws * args.steps / e2e_s
    e2e_equal = bool(np.array_equal(ctx.state()["position"], ctx_e2e.state()["position"]))
    ctx_e2e.close()

    # --- roofline of the dominant kernel family (timed on the twin context
    # over the same step indices) and of the narrow phase
    peak, peak_kind = measured_peaks()

    def family_roof(i):
        return {"kernel": FAMILIES[i], "bound": "hbm", "unit": "GB/s", "peak": peak, "peak_kind": peak_kind,
                "ms_per_launch": float(prof_ms[i] / max(prof_n[i], 1)), "launches": int(prof_n[i]),
                "share_of_step_time": float(prof_ms[i] / max(prof_ms.sum(), 1e-30)), "traffic": None}

    n_joints = int(sc.joint_type.shape[0])
    newton_iters = int(sum(d["newton_iterations"] for d in prof_steps))
    mean_contacts = float(np.mean([d["n_contacts"] for d in prof_steps]))
    traffic = ncu_traffic()
    roof_newton = family_roof(FAMILIES.index("newton"))
    roof_newton["traffic"] = traffic.get("k_newton")
    nb = newton_bytes(sc.n_bodies, n_joints, mean_contacts)
    ach = nb * newton_iters / (prof_ms[FAMILIES.index("newton")] / 1e3) / 1e9
    roof_newton.update(achieved=ach, frac=ach / peak, algorithmic_bytes_per_newton_iteration=nb,
                       newton_iterations=newton_iters,
                       note=("latency-bound: one Newton solve per ALM iteration on a 16-CTA thread-block cluster "
                             "(hardware cluster barrier); phases wait on latency chains (joint Jacobians, trial "
                             "energies, one-warp factorisation of the hopper's star component); under 1 MB of DRAM "
                             "per launch, HBM is not the limiter"))
    roof_narrow = family_roof(FAMILIES.index("narrow_phase"))
    roof_narrow["traffic"] = traffic.get("k_narrow_rows")
    if cand_counts:
        fv, ee = cand_counts
        # a detection pass is 4 launches (FV+EE rows, their hit emission, and
        # the gated VV rows / emission); count the pass as one unit
        passes = prof_n[FAMILIES.index("narrow_phase")] / 4.0
        secs = prof_ms[FAMILIES.index("narrow_phase")] / 1e3
        bytes_pass = staged_pair_bytes(diag["n_body_pairs"], diag["n_contacts"])
        per_cand = candidate_operand_bytes(fv, ee, diag["n_contacts"])
        ach = bytes_pass * passes / secs / 1e9
        roof_narrow.update(achieved=ach, frac=ach / peak, algorithmic_bytes_per_pass=bytes_pass,
                           per_candidate_operand_gbs=per_cand * passes / secs / 1e9,
                           note=("compute-bound: each pair's selected primitives are staged once and every "
                                 "candidate is tested from registers / shared memory (ncu: FP64 pipe ~40 % "
                                 "active); per_candidate_operand_gbs counts every candidate's operands"))
    # FP64 roofline of the narrow phase against this device's measured DFMA
    # throughput.  Algorithmic FP64 operations of the common path per item:
    # a face-vertex item 8 (p - v0, the dot with the face normal; the
    # barycentric test runs only inside dhat), an edge-edge item 12 (midpoint
    # difference, its squared length, the sum of the radii and its square;
    # the closest-point solve runs only inside the bounding spheres).  The
    # kernels keep every multiply and add separately rounded (bit parity with
    # the CPU path), so 0.5 of the FMA peak is their ceiling.
    fp64_tflops, fp64_ms = runtime.fp64_peak(stream.cuda_stream)
    roof_fp64 = None
    if cand_counts:
        fv, ee = cand_counts
        passes = prof_n[FAMILIES.index("narrow_phase")] / 4.0
        secs = prof_ms[FAMILIES.index("narrow_phase")] / 1e3
        flops_pass = 8.0 * fv + 12.0 * ee
        ach_tf = flops_pass * passes / secs / 1e12
        roof_fp64 = {"kernel": "narrow_phase", "bound": "fp64", "unit": "TFLOP/s", "peak": fp64_tflops,
                     "peak_kind": "measured (nxd_fp64_peak: DFMA chains on every SM, best of 5)",
                     "achieved": ach_tf, "frac": ach_tf / fp64_tflops, "flops_per_pass": flops_pass,
                     "fv_items": int(fv), "ee_items": int(ee),
                     "note": ("common-path FP64 operations of every face-vertex (8) and edge-edge (12) item over the "
                              "family's time (rows + emission launches); no FMA contraction, so 0.5 is the ceiling")}
    fam = int(np.argmax(prof_ms))
    roof = roof_newton if FAMILIES[fam] == "newton" else (roof_narrow if FAMILIES[fam] == "narrow_phase"
                                                          else dict(family_roof(fam), achieved=None, frac=None))
    per_family = {FAMILIES[i]: {"ms": round(float(prof_ms[i]), 3), "launches": int(prof_n[i])} for i in range(9)}

    full = full_run_leg(torch, lib, stream, flush)

    mode_i = None if args.no_mode_i else mode_i_leg(ctx, sc)
    if mode_i is not None:
        mode_i["step"] = ipc_step_leg()
        mode_i["step_pcg"] = ipc_step_leg(solver=1)
        mode_i["step_64"] = ipc_step_leg(n_cubes=64, columns=16, settle=30, steps=10)
        mode_i["step_bowl"] = ipc_step_leg(settle=0, steps=40, bowl=True)
        mode_i["step_bowl_friction"] = ipc_step_leg(settle=0, steps=20, bowl=True, mu=0.3)

    batched = None
    if not args.no_batched:
        batched = batched_leg(torch, min(args.steps, 10), 2, flush, ws, rank)
    diffl = None if args.no_diff else diff_leg(torch)
    pcg = None if args.no_pcg else pcg_leg()
    adj = None if args.no_diff else adjoint_leg(torch, args.adjoint_sets)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        walls, ff = oracle_steps(scenes.hopper_chains, threads, args.warmup, 1, literal=True)
        cpu = {"value": 1.0 / walls[0], "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"step {args.warmup + 1} (the first timed index) of the same scene through the CPU oracle "
                          f"(the reference's step restated; the reference itself cannot be built here) on "
                          f"{threads} threads with the reference's literal computeSceneMinDistance, timed whole: "
                          f"{walls[0]:.1f} s; steps 1-{args.warmup} fast-forwarded untimed ({ff:.1f} s)")}
        if mode_i is not None:
            mode_i["step"]["cpu_baseline"] = ipc_step_cpu_baseline(8, 1, 30, 20)
            mode_i["step_64"]["cpu_baseline"] = ipc_step_cpu_baseline(64, 16, 30, 10)
            mode_i["step_bowl"]["cpu_baseline"] = ipc_step_cpu_baseline(0, 0, 0, 2, bowl=True)
            mode_i["step_bowl_friction"]["cpu_baseline"] = ipc_step_cpu_baseline(0, 0, 0, 1, bowl=True, mu=0.3)
    launches_total = int(timed_n.sum())
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "batched_scene_steps_per_s": None if batched is None else batched["value"],
                   "batched_over_plain": None if batched is None else batched["batched_over_plain"],
                   "batched_groups": None if batched is None else batched["groups"],
                   "adjoint_fwd_plus_adj_over_fwd": None if adj is None else adj["fwd_plus_adj_over_fwd"],
                   "full_run_steps_per_s": full["steps_per_s"],
                   "mode_i_bowl_steps_per_s": None if mode_i is None else mode_i["step_bowl"]["steps_per_s"],
                   "replicas": ws, "l2": "flushed between steps (256 MiB write, untimed)",
                   "timing": ("value: K steps, each the step's CUDA graph, CUDA events per step; per_family_ms and "
                              "roofline: the same K step indices on a twin context of the same scene with CUDA "
                              "events around every launch; e2e: the same K step indices on a third context "
                              "(same warm-up), each nxd_set_state from pinned host memory, nxd_step, "
                              "nxd_get_state back, wall clock"),
                   "twin_state_equal": twin_equal,
                   "e2e_state_equal": e2e_equal,
                   "fp64_peak_tflops": fp64_tflops,
                   "full_run_steps": full["steps"],
                   "full_run_ms_max_step": full["ms_max_step"],
                   "full_run": full,
                   "per_family_ms": per_family, "last_step": {k: diag[k] for k in
                                                              ("n_body_pairs", "n_contacts", "alm_iterations",
                                                               "newton_iterations", "status")},
                   "batched": batched,
                   "diff": diffl,
                   "adjoint": adj,
                   "pcg": pcg,
                   "mode_i": mode_i},
        "roofline": roof,
        "roofline_narrow_phase": roof_narrow,
        "roofline_fp64_narrow_phase": roof_fp64,
        "roofline_pcg": None if pcg is None else {
            "kernel": "k_pcg", "bound": "hbm", "unit": "GB/s", "peak": peak, "peak_kind": peak_kind,
            "achieved": pcg["achieved_gbs"], "frac": pcg["achieved_gbs"] / peak if pcg["achieved_gbs"] else None,
            "traffic": ncu_traffic().get("k_pcg"), "bytes_per_iteration": pcg["bytes_per_iteration"],
            "note": ("block-Jacobi PCG, one cooperative kernel; the block product streams the 400 MB matrix each "
                     "iteration; traffic: ncu DRAM bytes per iteration")},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches_total,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    ctx_prof.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
