"""Batched IK over robots of uneven size: one persistent work-queue launch.

``MixedIkBatch`` solves many IK problems of several robot classes (chains,
trees, different DOF and sphere counts, one or several end effectors) that
share one obstacle world.  It lays every class's seeds and outputs out as
``[problems, seed_stride, n_act]`` so each problem can carry its own seed
count, cuts the problems into work items ``(class, problem, first seed,
count)`` sorted longest first, and runs them through ``pk_ik_batch``: one
persistent kernel per body (the seed-group kernel for small single-EE
robots, the warp-per-seed kernel for the rest) whose blocks pull items from
a device counter until the list is empty.  The per-class FP64 verification
and winner selection (``pk_ik_verify_select``) follow on the same stream.
The whole solve can be captured once in a CUDA graph and replayed; an
autotuner picks the seed-group kernel's lanes per seed and seeds per block
the warp body's lanes per seed and the obstacle tile (the per-block obstacle
grid's cells per axis) by timing the actual batch.

It is the persistent form of calling ``ls_ik_solve_cuda_batch``
(``src/pyroffi/optimization_engines/_ls_ik.py:1002-1172``) once per robot
class with every problem padded to the largest seed count.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .ik import BatchIkSolver

BODY_SEED_GROUP, BODY_WARP, BODY_SEED_GROUP16 = 0, 1, 2


@dataclass
class ClassResult:
    winner_cfg: torch.Tensor   # [P_c, n_act]
    pos_err: torch.Tensor      # [P_c] float64
    rot_err: torch.Tensor      # [P_c] float64
    success: torch.Tensor      # [P_c] int32


def default_body(n_act: int, n_ee: int) -> int:
    """Register kernels where they fit: the 8-wide seed-group body for small
    single-EE robots, the 16-wide one-lane body up to 16 DOF and 2 EEs, the
    warp-per-seed body beyond."""
    if n_act <= 8 and n_ee == 1:
        return BODY_SEED_GROUP
    if n_act <= 16 and n_ee <= 2:
        return BODY_SEED_GROUP16
    return BODY_WARP


class MixedIkBatch:
    """classes: objects with ``model``, ``spheres`` and ``target_links`` (e.g.
    ``workloads.MixedIkClass``); ``world``: the shared obstacles."""

    def __init__(self, classes, world, *, max_iter: int = 30, lambda_init: float = 1e-2,
                 lambda_down: float = 0.1, lambda_up: float = 10.0, pos_weight: float = 50.0,
                 ori_weight: float = 10.0, collision_weight: float = 1e4, collision_margin: float = 0.02,
                 pos_tol: float = 1e-3, rot_tol: float = 1e-2, threads_per_seed: int = 0,
                 seeds_per_block: int = 0, lanes_per_wide_seed: int = 0, bodies=None, blocks: int = 0,
                 device="cuda"):
        self.device = torch.device(device)
        self.classes = list(classes)
        if not 1 <= len(self.classes) <= 8:
            raise ValueError("MixedIkBatch takes 1 to 8 robot classes")
        opts = dict(max_iter=max_iter, lambda_init=lambda_init, lambda_down=lambda_down, lambda_up=lambda_up,
                    pos_weight=pos_weight, ori_weight=ori_weight, collision_weight=collision_weight,
                    collision_margin=collision_margin, pos_tol=pos_tol, rot_tol=rot_tol, device=self.device)
        self.solvers = [BatchIkSolver(c.model, c.target_links, spheres=c.spheres, world=world, **opts)
                        for c in self.classes]
        self.world = self.solvers[0].world
        coll = any(int(s.opt.enable_collision) for s in self.solvers)
        self.opt = _lib.LmOptions(max_iter, pos_weight, ori_weight, lambda_init, lambda_down, lambda_up,
                                  1e-8, 1e-8, int(coll), collision_weight, collision_margin,
                                  threads_per_seed, seeds_per_block, lanes_per_wide_seed)
        self.bodies = list(bodies) if bodies is not None else [
            default_body(c.model.n_act, s.n_ee) for c, s in zip(self.classes, self.solvers)]
        self.blocks = blocks
        self.queue = torch.zeros(2, dtype=torch.int32, device=self.device)
        self._graph = None
        self._desc = None

    # -- layout -------------------------------------------------------------
    def prepare(self, problem_class: np.ndarray, n_seeds: np.ndarray) -> None:
        """Allocate the per-class buffers and build the work items for
        problems of classes ``problem_class`` with ``n_seeds`` seeds each
        (problem p is row ``index_in_class[p]`` of its class's buffers, in
        order of appearance)."""
        problem_class = np.asarray(problem_class, np.int64)
        n_seeds = np.asarray(n_seeds, np.int64)
        self.problem_class, self.n_seeds = problem_class, n_seeds
        dev = self.device
        self.counts, self.strides = [], []
        self.index_in_class = np.zeros(len(problem_class), np.int64)
        self.targets, self.seeds, self.out_cfg, self.out_err = [], [], [], []
        for c, (cl, s) in enumerate(zip(self.classes, self.solvers)):
            idx = np.nonzero(problem_class == c)[0]
            self.index_in_class[idx] = np.arange(len(idx))
            Pc = len(idx)
            stride = int(n_seeds[idx].max()) if Pc else 0
            n = cl.model.n_act
            self.counts.append(Pc)
            self.strides.append(stride)
            self.targets.append(torch.zeros((Pc, s.n_ee, 7), dtype=torch.float32, device=dev))
            self.seeds.append(torch.zeros((Pc, stride, n), dtype=torch.float32, device=dev))
            self.out_cfg.append(torch.zeros((Pc, stride, n), dtype=torch.float32, device=dev))
            # unused seed slots are never written, so they never win the selection
            self.out_err.append(torch.full((Pc, stride), float("inf"), dtype=torch.float32, device=dev))
        self._build_items()
        self._graph = None

    def _chunk(self, c: int) -> int:
        """Seeds per item: one block's seeds for the seed-group bodies (the
        library's defaults: one lane x 128 seeds for the 8-wide body, one
        lane x 96 seeds for the 16-wide body), 64 for the warp body."""
        if self.bodies[c] == BODY_SEED_GROUP:
            tps = self.opt.threads_per_seed if self.opt.threads_per_seed > 0 else 1
            if self.opt.seeds_per_block > 0:
                return self.opt.seeds_per_block
            return 128 if self.opt.threads_per_seed <= 0 else 128 // tps
        if self.bodies[c] == BODY_SEED_GROUP16:
            return 96
        return 64

    def _cost_per_seed(self, c: int) -> float:
        """Relative per-seed cost for the longest-first order: FK joints,
        sphere tests and the solve size."""
        s, m = self.solvers[c], self.classes[c].model
        n_rs = int(s.spheres_local.shape[0])
        return m.n_joints * 8 + n_rs * 6 + m.n_act ** 2 + (200 if self.bodies[c] != BODY_SEED_GROUP else 0)

    def _build_items(self) -> None:
        items, cost = [], []
        for p, c in enumerate(self.problem_class):
            ch = self._chunk(int(c))
            i = int(self.index_in_class[p])
            total = int(self.n_seeds[p])
            w = self._cost_per_seed(int(c))
            for first in range(0, total, ch):
                cnt = min(ch, total - first)
                items.append((int(c), i, first, cnt))
                cost.append(w * cnt)
        order = np.argsort(-np.asarray(cost, np.float64), kind="stable")
        arr = np.asarray(items, np.int32).reshape(-1, 4)[order]
        self.items = torch.as_tensor(np.ascontiguousarray(arr), device=self.device)
        self.n_items = int(arr.shape[0])
        self._desc = None

    def _descriptors(self):
        if self._desc is not None:
            return self._desc
        arr = (_lib.IkClass * len(self.classes))()
        for c, (cl, s) in enumerate(zip(self.classes, self.solvers)):
            r = s.robot
            d = arr[c]
            (d.twists, d.parent_tf, d.parent_idx, d.act_idx, d.mimic_mul, d.mimic_off, d.mimic_act_idx,
             d.topo_inv) = [ptr(t) for t in r.fk_args()]
            d.n_joints, d.n_act = cl.model.n_joints, cl.model.n_act
            d.target_jnts, d.ancestor_masks, d.target_Ts = ptr(s.target_jnts), ptr(s.ancestor_masks), ptr(self.targets[c])
            d.n_ee = s.n_ee
            d.robot_spheres_local, d.robot_sphere_joint_idx = ptr(s.spheres_local), ptr(s.sphere_joint)
            d.n_robot_spheres = int(s.spheres_local.shape[0])
            d.self_i, d.self_j, d.n_self = ptr(s.self_i), ptr(s.self_j), int(s.self_i.shape[0])
            d.lower, d.upper, d.fixed_mask = ptr(r.lower), ptr(r.upper), ptr(s.fixed_mask)
            d.seeds, d.out_cfg, d.out_err = ptr(self.seeds[c]), ptr(self.out_cfg[c]), ptr(self.out_err[c])
            d.n_problems, d.seed_stride = self.counts[c], self.strides[c]
            d.body = self.bodies[c]
        self._desc = arr
        return arr

    # -- solve --------------------------------------------------------------
    def load(self, targets, seeds) -> None:
        """Copy per-class targets ``[P_c, n_ee, 7]`` (or ``[P_c, 7]``) and
        seeds ``[P_c, >= used seeds, n_act]`` into the batch buffers."""
        for c in range(len(self.classes)):
            if self.counts[c] == 0:
                continue
            t = f32(torch.as_tensor(targets[c])).to(self.device).reshape(self.targets[c].shape)
            self.targets[c].copy_(t, non_blocking=True)
            sd = f32(torch.as_tensor(seeds[c])).to(self.device)
            self.seeds[c].copy_(sd[:, : self.strides[c]], non_blocking=True)

    def run_lm(self) -> None:
        """The batched LM launch(es) on the current stream."""
        Ms, Mc, Mb, Mh = self.world.counts()
        _lib.call("pk_ik_batch", stream_ptr(self.device), ctypes.byref(self.opt), ctypes.cast(self._descriptors(),
                  ctypes.c_void_p), len(self.classes), *[ptr(t) for t in self.world.arrays()], Ms, Mc, Mb, Mh,
                  ptr(self.items), self.n_items, ptr(self.queue), int(self.blocks))

    def verify(self) -> list[ClassResult]:
        out = []
        for c, s in enumerate(self.solvers):
            if self.counts[c] == 0:
                out.append(None)
                continue
            w, pos, rot, ok = s.verify_select(self.out_cfg[c], self.out_err[c], self.targets[c])
            out.append(ClassResult(w, pos, rot, ok))
        return out

    def solve(self) -> list[ClassResult]:
        if self._graph is not None:
            self._graph.replay()
            return self._graph_out
        self.run_lm()
        return self.verify()

    def launches_per_solve(self) -> int:
        """Kernels per solve: one persistent launch per body in use, one
        verification per class."""
        bodies = {self.bodies[c] for c in range(len(self.classes)) if self.counts[c]}
        return len(bodies) + sum(1 for c in range(len(self.classes)) if self.counts[c])

    def capture(self) -> None:
        """Capture LM + verification once in a CUDA graph; later ``solve()``
        calls replay it on the buffers filled by ``load``."""
        self._graph = None
        self.run_lm()
        self.verify()
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="relaxed"):
            self.run_lm()
            self._graph_out = self.verify()
        self._graph = g

    # -- autotuning ---------------------------------------------------------
    def autotune(self, candidates=((1, 128), (1, 64), (2, 64), (4, 32)), wide_lanes=(16, 32), grids=(0, 4, 6),
                 reps: int = 2):
        """Time the prepared batch for each (threads_per_seed, seeds_per_block)
        of the 8-wide seed-group body, each lane count per seed of the warp
        body and each obstacle tile (``obstacle_grid``: the cells per axis of
        the per-block obstacle grid, 0 = the default, -1 = none), and keep
        the fastest.  The item list is rebuilt for each, since a seed-group
        item holds one block's seeds.  Returns {(threads_per_seed,
        seeds_per_block, lanes_per_wide_seed, obstacle_grid): ms}."""
        used = {b for c, b in enumerate(self.bodies) if self.counts[c]}
        if BODY_SEED_GROUP not in used:
            candidates = ((self.opt.threads_per_seed, self.opt.seeds_per_block),)
        if BODY_WARP not in used:
            wide_lanes = (self.opt.lanes_per_wide_seed,)
        results = {}
        for tps, spb in candidates:
            for lanes in wide_lanes:
                for grid in grids:
                    self.opt.threads_per_seed, self.opt.seeds_per_block = tps, spb
                    self.opt.lanes_per_wide_seed, self.opt.obstacle_grid = lanes, grid
                    self._build_items()
                    self.run_lm()
                    torch.cuda.synchronize(self.device)
                    ts = []
                    for _ in range(reps):
                        t0 = time.perf_counter()
                        self.run_lm()
                        torch.cuda.synchronize(self.device)
                        ts.append(time.perf_counter() - t0)
                    results[(tps, spb, lanes, grid)] = 1e3 * min(ts)
        tps, spb, lanes, grid = min(results, key=results.get)
        self.opt.threads_per_seed, self.opt.seeds_per_block = tps, spb
        self.opt.lanes_per_wide_seed, self.opt.obstacle_grid = lanes, grid
        self._build_items()
        self._graph = None
        return results
