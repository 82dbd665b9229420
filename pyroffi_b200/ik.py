"""Batched multi-seed LM IK on the GPU (torch tensors, sm_100a kernels).

``BatchIkSolver`` mirrors the reference's batched CUDA driver
``ls_ik_solve_cuda_batch`` / ``_ls_ik_solve_cuda_batch_jit``
(``src/pyroffi/optimization_engines/_ls_ik.py:879-1172``): seed generation
(half warm starts ``clip(prev + 0.05 N(0,1))``, half uniform in the limits),
one LM launch over every (problem, seed), then the per-problem winner
``argmin(err + continuity * ||q - prev||^2)``.  Two additions: explicit
robot-sphere self-collision pairs in the LM penalty, and an FP64
re-verification of every winner's pose error (success = position < pos_tol
and rotation < rot_tol).  One solve is two kernel launches
(``pk_ls_ik_ex``, ``pk_ik_verify_select``).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .device import DeviceRobot, DeviceWorld
from .robot import RobotModel, RobotSpheres


@dataclass
class IkResult:
    winner_cfg: torch.Tensor    # [P, n_act]
    pos_err: torch.Tensor       # [P] float64, FP64 FK of the winner
    rot_err: torch.Tensor       # [P] float64
    success: torch.Tensor       # [P] int32
    cfgs: torch.Tensor          # [P, Sd, n_act] best config per seed
    errs: torch.Tensor          # [P, Sd] its weighted error


class BatchIkSolver:
    def __init__(self, model: RobotModel, target_links, *, spheres: RobotSpheres | None = None,
                 world=None, self_pairs: np.ndarray | None = None, max_iter: int = 60,
                 pos_weight: float = 50.0, ori_weight: float = 10.0, lambda_init: float = 5e-3,
                 lambda_down: float = 0.5, lambda_up: float = 3.0, eps_pos: float = 1e-8,
                 eps_ori: float = 1e-8, collision_weight: float = 1e4,
                 collision_margin: float = 0.02, pos_tol: float = 1e-3, rot_tol: float = 1e-2,
                 threads_per_seed: int = 0, seeds_per_block: int = 0, fp64_solve: bool = False, device="cuda"):
        self.device = torch.device(device)
        self.model = model
        self.robot = DeviceRobot.upload(model, self.device)
        self.target_links = tuple(int(x) for x in (target_links if np.ndim(target_links) else [target_links]))
        self.n_ee = len(self.target_links)
        tj = np.asarray([model.link_joint(l) for l in self.target_links], np.int32)
        anc = np.stack([model.ancestor_mask(l) for l in self.target_links]).astype(np.int32)
        self.target_jnts = torch.as_tensor(tj, device=self.device)
        self.ancestor_masks = torch.as_tensor(anc, device=self.device)
        if spheres is not None:
            rs, jidx, _ = spheres.flat_for_ik(model)
        else:
            rs, jidx = np.zeros((0, 4), np.float32), np.zeros((0,), np.int32)
        self.spheres_local = torch.as_tensor(rs, device=self.device)
        self.sphere_joint = torch.as_tensor(jidx, device=self.device)
        from .workloads import empty_world
        self.world = DeviceWorld.upload(world if world is not None else empty_world(), self.device)
        sp = np.zeros((0, 2), np.int32) if self_pairs is None else np.asarray(self_pairs, np.int32).reshape(-1, 2)
        self.self_i = torch.as_tensor(np.ascontiguousarray(sp[:, 0]), device=self.device)
        self.self_j = torch.as_tensor(np.ascontiguousarray(sp[:, 1]), device=self.device)
        self.fixed_mask = torch.zeros(model.n_act, dtype=torch.int32, device=self.device)
        coll = (rs.shape[0] > 0) and (sum(self.world.counts()) > 0 or sp.shape[0] > 0)
        self.opt = _lib.LmOptions(max_iter, pos_weight, ori_weight, lambda_init, lambda_down, lambda_up,
                                  eps_pos, eps_ori, int(coll), collision_weight, collision_margin,
                                  threads_per_seed, seeds_per_block, 0, int(fp64_solve))
        self.pos_tol, self.rot_tol = pos_tol, rot_tol

    def set_fixed_mask(self, mask) -> None:
        self.fixed_mask = torch.as_tensor(np.asarray(mask, np.int32), device=self.device)

    def make_seeds(self, previous_cfgs: torch.Tensor, num_seeds: int,
                   generator: torch.Generator | None = None) -> torch.Tensor:
        """Half warm starts ``clip(prev + 0.05 N(0,1))``, half uniform in the
        limits; fixed joints keep ``prev`` (``_ls_ik.py:920-938``)."""
        P = previous_cfgs.shape[0]
        n = self.model.n_act
        lo, hi = self.robot.lower, self.robot.upper
        n_warm = max(1, num_seeds // 2)
        n_rand = num_seeds - n_warm
        prev = f32(previous_cfgs).to(self.device)
        warm = prev[:, None, :] + 0.05 * torch.randn((P, n_warm, n), device=self.device, generator=generator)
        warm = torch.minimum(torch.maximum(warm, lo), hi)
        rnd = lo + (hi - lo) * torch.rand((P, n_rand, n), device=self.device, generator=generator)
        seeds = torch.cat([warm, rnd], dim=1)
        fixed = self.fixed_mask.bool()[None, None, :]
        return torch.where(fixed, prev[:, None, :], seeds).contiguous()

    def run_lm(self, target_T: torch.Tensor, seeds: torch.Tensor):
        """LM over all (problem, seed): returns (cfgs [P,Sd,n], errs [P,Sd])."""
        P, Sd, n = (int(x) for x in seeds.shape)
        tgt = f32(target_T).reshape(P, self.n_ee, 7)
        s = f32(seeds)
        out_cfg = torch.empty((P, Sd, n), dtype=torch.float32, device=self.device)
        out_err = torch.empty((P, Sd), dtype=torch.float32, device=self.device)
        r = self.robot
        Ms, Mc, Mb, Mh = self.world.counts()
        _lib.call("pk_ls_ik_ex", stream_ptr(self.device), ctypes.byref(self.opt), ptr(s),
                  *[ptr(t) for t in r.fk_args()], ptr(self.target_jnts), ptr(self.ancestor_masks),
                  ptr(tgt), ptr(self.spheres_local), ptr(self.sphere_joint),
                  *[ptr(t) for t in self.world.arrays()], ptr(self.self_i), ptr(self.self_j),
                  ptr(r.lower), ptr(r.upper), ptr(self.fixed_mask), ptr(out_cfg), ptr(out_err),
                  P, Sd, n, self.model.n_joints, self.n_ee, int(self.spheres_local.shape[0]),
                  Ms, Mc, Mb, Mh, int(self.self_i.shape[0]))
        return out_cfg, out_err

    def verify_select(self, cfgs, errs, target_T, prev=None, continuity_weight: float = 0.0):
        P, Sd, n = (int(x) for x in cfgs.shape)
        tgt = f32(target_T).reshape(P, self.n_ee, 7)
        winner = torch.empty((P, n), dtype=torch.float32, device=self.device)
        pos = torch.empty(P, dtype=torch.float64, device=self.device)
        rot = torch.empty(P, dtype=torch.float64, device=self.device)
        ok = torch.empty(P, dtype=torch.int32, device=self.device)
        pv = f32(prev).to(self.device) if prev is not None else None
        r = self.robot
        _lib.call("pk_ik_verify_select", stream_ptr(self.device), ptr(cfgs), ptr(errs), ptr(pv),
                  float(continuity_weight), *[ptr(t) for t in r.fk_args()], ptr(self.target_jnts),
                  ptr(tgt), float(self.pos_tol), float(self.rot_tol), ptr(winner), ptr(pos), ptr(rot),
                  ptr(ok), P, Sd, n, self.model.n_joints, self.n_ee)
        return winner, pos, rot, ok

    def solve(self, target_T: torch.Tensor, seeds: torch.Tensor, prev=None,
              continuity_weight: float = 0.0) -> IkResult:
        cfgs, errs = self.run_lm(target_T, seeds)
        w, pos, rot, ok = self.verify_select(cfgs, errs, target_T, prev, continuity_weight)
        return IkResult(w, pos, rot, ok, cfgs, errs)


def ls_ik_solve_batch(model: RobotModel, target_link_indices, target_poses: torch.Tensor,
                      previous_cfgs: torch.Tensor, *, num_seeds: int = 32,
                      generator: torch.Generator | None = None, continuity_weight: float = 0.0,
                      spheres: RobotSpheres | None = None, world=None, **options) -> torch.Tensor:
    """Functional form of ``ls_ik_solve_cuda_batch``: target poses
    ``[P, 7]`` (single EE) or ``[P, n_ee, 7]`` -> winners ``[P, n_act]``."""
    solver = BatchIkSolver(model, target_link_indices, spheres=spheres, world=world,
                           device=target_poses.device, **options)
    seeds = solver.make_seeds(previous_cfgs, num_seeds, generator)
    return solver.solve(target_poses, seeds, prev=previous_cfgs,
                        continuity_weight=continuity_weight).winner_cfg
