"""HJCD-IK on the GPU (coarse coordinate descent + LM refinement).

Drop-in for ``hjcd_solve_cuda_batch`` and ``hjcd_solve_cuda``
(``src/pyroffi/optimization_engines/_hjcd_ik.py:655-830, 1069-1417``) over
``pk_hjcd_ik_coarse_cuda`` and ``pk_hjcd_ik_lm_cuda``:

1. seeds per problem: ``min(top_k, num_seeds)`` warm starts
   ``clip(prev + 0.05 N(0, 1))`` and uniform draws in the limits for the rest;
   fixed joints keep ``prev`` (``:1117-1131``);
2. the coarse kernel on every seed;
3. per problem, the ``top_k`` lowest coarse errors (ties to the lower seed
   index) repeated ``repeats`` times; every copy after the first ``top_k`` is
   perturbed by ``0.15 (upper - lower) N(0, 1)`` and clipped, fixed joints
   unperturbed (``:1163-1175``); ``(top_k, repeats)`` follow
   ``_get_refine_schedule`` (``:368-381``);
4. Gaussian kick noise ``[P, top_k * repeats, lm_max_iter, n]`` and the LM
   kernel;
5. the winner ``argmin(err + continuity_weight |q - prev|^2)`` per problem.

Random numbers come from a ``torch.Generator`` (the reference draws from
``jax.random``), so runs are reproducible here but not bit-identical to the
reference's draws.  Constraint callables and the post-hoc constraint LM of
the reference are not taken.
"""

from __future__ import annotations


import numpy as np
import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .device import DeviceRobot, DeviceWorld
from .robot import RobotModel, RobotSpheres

STALL_PATIENCE = 6


def refine_schedule(num_seeds: int) -> tuple[int, int]:
    """(top_k, repeats) of the refinement for a coarse batch of ``num_seeds``."""
    if num_seeds <= 8:
        return num_seeds, 24
    if num_seeds <= 16:
        return max(1, num_seeds // 2), 16
    if num_seeds <= 128:
        return max(1, int(num_seeds * 0.2)), 5
    if num_seeds <= 1024:
        return max(1, int(num_seeds * 0.02)), 5
    if num_seeds <= 2048:
        return max(1, int(num_seeds * 0.01)), 5
    return max(1, int(num_seeds * 0.01)), 2


def make_seeds(prev: torch.Tensor, lower: torch.Tensor, upper: torch.Tensor, fixed: torch.Tensor, num_seeds: int,
               n_warm: int, generator: torch.Generator | None = None) -> torch.Tensor:
    P, n = prev.shape
    warm = prev[:, None, :] + 0.05 * torch.randn((P, n_warm, n), device=prev.device, generator=generator)
    warm = torch.clamp(warm, lower, upper)
    rnd = lower + (upper - lower) * torch.rand((P, num_seeds - n_warm, n), device=prev.device, generator=generator)
    seeds = torch.cat([warm, rnd], dim=1)
    return torch.where(fixed.bool()[None, None, :], prev[:, None, :], seeds).contiguous()


def select_refine_seeds(cfg: torch.Tensor, err: torch.Tensor, top_k: int, repeats: int, lower: torch.Tensor,
                        upper: torch.Tensor, fixed: torch.Tensor,
                        generator: torch.Generator | None = None) -> torch.Tensor:
    """[P, top_k * repeats, n]: the top_k lowest-error configurations, then
    perturbed copies."""
    P, S, n = cfg.shape
    order = torch.sort(err, dim=1, stable=True).indices[:, :top_k]
    top = torch.gather(cfg, 1, order[:, :, None].expand(P, top_k, n))
    base = top.repeat(1, repeats, 1)
    noise = torch.randn((P, top_k * repeats, n), device=cfg.device, generator=generator) * (0.15 * (upper - lower))
    noise = torch.where(fixed.bool()[None, None, :], torch.zeros_like(noise), noise)
    original = (torch.arange(top_k * repeats, device=cfg.device) < top_k)[None, :, None]
    return torch.where(original, base, torch.clamp(base + noise, lower, upper)).contiguous()


def pick_winner(cfg: torch.Tensor, err: torch.Tensor, prev: torch.Tensor, continuity_weight: float):
    """Per problem the configuration minimising err + w |q - prev|^2 (ties to the lowest index)."""
    score = err + continuity_weight * torch.sum((cfg - prev[:, None, :]) ** 2, dim=-1)
    best = torch.argmin(score, dim=1)
    P = cfg.shape[0]
    return cfg[torch.arange(P, device=cfg.device), best], score[torch.arange(P, device=cfg.device), best]


class HjcdSolver:
    def __init__(self, model: RobotModel, target_links, *, spheres: RobotSpheres | None = None, world=None,
                 enable_collision: bool = False, collision_weight: float = 1e4, collision_margin: float = 0.02,
                 device="cuda"):
        self.device = torch.device(device)
        self.model = model
        self.robot = DeviceRobot.upload(model, self.device)
        links = tuple(int(x) for x in (target_links if np.ndim(target_links) else [target_links]))
        self.n_ee = len(links)
        self.target_jnts = torch.as_tensor(np.asarray([model.link_joint(l) for l in links], np.int32),
                                           device=self.device)
        self.ancestor_masks = torch.as_tensor(np.stack([model.ancestor_mask(l) for l in links]).astype(np.int32),
                                              device=self.device)
        if spheres is not None:
            rs, jidx, _ = spheres.flat_for_ik(model)
        else:
            rs, jidx = np.zeros((0, 4), np.float32), np.zeros((0,), np.int32)
        self.spheres_local = torch.as_tensor(rs, device=self.device)
        self.sphere_joint = torch.as_tensor(jidx, device=self.device)
        from .workloads import empty_world
        self.world = DeviceWorld.upload(world if world is not None else empty_world(), self.device)
        self.enable_collision = bool(enable_collision)
        self.collision_weight, self.collision_margin = float(collision_weight), float(collision_margin)
        self.fixed_mask = torch.zeros(model.n_act, dtype=torch.int32, device=self.device)

    def set_fixed_mask(self, mask) -> None:
        self.fixed_mask = torch.as_tensor(np.asarray(mask, np.int32), device=self.device)

    def _common(self):
        r = self.robot
        return [*[ptr(t) for t in r.fk_args()], ptr(self.target_jnts), ptr(self.ancestor_masks)]

    def _tail(self):
        return [ptr(self.spheres_local), ptr(self.sphere_joint), *[ptr(t) for t in self.world.arrays()],
                ptr(self.robot.lower), ptr(self.robot.upper), ptr(self.fixed_mask)]

    def _extents(self, P, S):
        return [P, S, self.model.n_act, self.model.n_joints, self.n_ee, int(self.spheres_local.shape[0]),
                *self.world.counts()]

    def coarse(self, seeds: torch.Tensor, target_T: torch.Tensor, k_max: int = 20):
        """-> (cfg [P, S, n], err [P, S])."""
        s = f32(seeds)
        P, S, n = (int(v) for v in s.shape)
        tgt = f32(target_T).reshape(P, self.n_ee, 7)
        out = torch.empty((P, S, n), dtype=torch.float32, device=self.device)
        err = torch.empty((P, S), dtype=torch.float32, device=self.device)
        _lib.call("pk_hjcd_ik_coarse_cuda", stream_ptr(self.device), ptr(s), *self._common(), ptr(tgt),
                  *self._tail(), int(k_max), int(self.enable_collision), self.collision_weight,
                  self.collision_margin, ptr(out), ptr(err), *self._extents(P, S))
        return out, err

    def refine(self, seeds: torch.Tensor, noise: torch.Tensor, target_T: torch.Tensor, *, max_iter: int = 40,
               stall_patience: int = STALL_PATIENCE, lambda_init: float = 5e-3, limit_prior_weight: float = 1e-3,
               kick_scale: float = 0.015, eps_pos: float = 1e-8, eps_ori: float = 1e-8):
        """-> (best cfg [P, S, n], err [P, S], stop [P])."""
        s = f32(seeds)
        P, S, n = (int(v) for v in s.shape)
        tgt = f32(target_T).reshape(P, self.n_ee, 7)
        nz = f32(noise)
        out = torch.empty((P, S, n), dtype=torch.float32, device=self.device)
        err = torch.empty((P, S), dtype=torch.float32, device=self.device)
        stop = torch.empty((P,), dtype=torch.int32, device=self.device)
        _lib.call("pk_hjcd_ik_lm_cuda", stream_ptr(self.device), ptr(s), ptr(nz), *self._common(), ptr(tgt),
                  *self._tail(), int(max_iter), int(stall_patience), float(lambda_init), float(limit_prior_weight),
                  float(kick_scale), float(eps_pos), float(eps_ori), int(self.enable_collision),
                  self.collision_weight, self.collision_margin, ptr(out), ptr(err), ptr(stop), *self._extents(P, S))
        return out, err, stop

    def solve(self, target_T: torch.Tensor, previous_cfgs: torch.Tensor, *, num_seeds: int = 32,
              coarse_max_iter: int = 20, lm_max_iter: int = 40, eps_pos: float = 1e-8, eps_ori: float = 1e-8,
              lambda_init: float = 5e-3, continuity_weight: float = 0.0, limit_prior_weight: float = 1e-3,
              kick_scale: float = 0.015, generator: torch.Generator | None = None, return_all: bool = False):
        """Best configuration per problem [P, n] (``hjcd_solve_cuda_batch``)."""
        prev = f32(previous_cfgs).to(self.device)
        P, n = prev.shape
        lo, hi, fx = self.robot.lower, self.robot.upper, self.fixed_mask
        top_k, repeats = refine_schedule(num_seeds)
        seeds = make_seeds(prev, lo, hi, fx, num_seeds, min(top_k, num_seeds), generator)
        ccfg, cerr = self.coarse(seeds, target_T, coarse_max_iter)
        lm_seeds = select_refine_seeds(ccfg, cerr, top_k, repeats, lo, hi, fx, generator)
        kicks = torch.randn((P, top_k * repeats, lm_max_iter, n), device=self.device, generator=generator)
        rcfg, rerr, _ = self.refine(lm_seeds, kicks, target_T, max_iter=lm_max_iter, lambda_init=lambda_init,
                                    limit_prior_weight=limit_prior_weight, kick_scale=kick_scale, eps_pos=eps_pos,
                                    eps_ori=eps_ori)
        best, score = pick_winner(rcfg, rerr, prev, continuity_weight)
        if return_all:
            return best, score, (seeds, ccfg, cerr, lm_seeds, kicks, rcfg, rerr)
        return best


def hjcd_solve_cuda_batch(model: RobotModel, target_links, target_T, previous_cfgs, **kw):
    """Functional form: builds an ``HjcdSolver`` and solves."""
    ctor = {k: kw.pop(k) for k in ("spheres", "world", "enable_collision", "collision_weight", "collision_margin",
                                   "device") if k in kw}
    s = HjcdSolver(model, target_links, **ctor)
    return s.solve(torch.as_tensor(target_T, device=s.device), torch.as_tensor(previous_cfgs, device=s.device), **kw)


__all__ = ["HjcdSolver", "hjcd_solve_cuda_batch", "refine_schedule", "make_seeds", "select_refine_seeds",
           "pick_winner", "STALL_PATIENCE"]
