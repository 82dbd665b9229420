"""SQP-IK on the GPU: joint limits as hard bounds on every step.

Drop-in for ``sqp_ik_solve_cuda_batch`` / ``sqp_ik_solve_cuda``
(``src/pyroffi/optimization_engines/_sqp_ik.py:409-530, 734-1005``) over
``pk_sqp_ik_cuda``:

1. seeds per problem: ``max(1, num_seeds // 2)`` warm starts
   ``clip(prev + 0.05 N(0, 1))`` and uniform draws in the limits for the rest;
   fixed joints keep ``prev`` (``:775-795``);
2. the SQP kernel on every (problem, seed);
3. the winner ``argmin(err + continuity_weight |q - prev|^2)`` per problem.

Random numbers come from a ``torch.Generator`` (the reference draws from
``jax.random``).  Constraint callables and the post-hoc constraint LM of the
reference are not taken.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .hjcd import HjcdSolver, make_seeds, pick_winner


class SqpSolver(HjcdSolver):
    """Same robot / collision setup as ``HjcdSolver``; ``run`` is the SQP kernel."""

    def run(self, seeds: torch.Tensor, target_T: torch.Tensor, *, max_iter: int = 60, n_inner_iters: int = 2,
            pos_weight: float = 50.0, ori_weight: float = 10.0, lambda_init: float = 5e-3, eps_pos: float = 1e-8,
            eps_ori: float = 1e-8):
        """-> (best cfg [P, S, n], weighted error [P, S])."""
        s = f32(seeds)
        P, S, n = (int(v) for v in s.shape)
        tgt = f32(target_T).reshape(P, self.n_ee, 7)
        out = torch.empty((P, S, n), dtype=torch.float32, device=self.device)
        err = torch.empty((P, S), dtype=torch.float32, device=self.device)
        _lib.call("pk_sqp_ik_cuda", stream_ptr(self.device), ptr(s), *self._common(), ptr(tgt), *self._tail(),
                  int(max_iter), int(n_inner_iters), float(pos_weight), float(ori_weight), float(lambda_init),
                  float(eps_pos), float(eps_ori), int(self.enable_collision), self.collision_weight,
                  self.collision_margin, ptr(out), ptr(err), *self._extents(P, S))
        return out, err

    def solve(self, target_T: torch.Tensor, previous_cfgs: torch.Tensor, *, num_seeds: int = 32,
              max_iter: int = 60, n_inner_iters: int = 2, pos_weight: float = 50.0, ori_weight: float = 10.0,
              lambda_init: float = 5e-3, eps_pos: float = 1e-8, eps_ori: float = 1e-8,
              continuity_weight: float = 0.0, generator: torch.Generator | None = None, return_all: bool = False):
        """Best configuration per problem [P, n] (``sqp_ik_solve_cuda_batch``)."""
        prev = f32(previous_cfgs).to(self.device)
        seeds = make_seeds(prev, self.robot.lower, self.robot.upper, self.fixed_mask, num_seeds,
                           max(1, num_seeds // 2), generator)
        cfg, err = self.run(seeds, target_T, max_iter=max_iter, n_inner_iters=n_inner_iters, pos_weight=pos_weight,
                            ori_weight=ori_weight, lambda_init=lambda_init, eps_pos=eps_pos, eps_ori=eps_ori)
        best, score = pick_winner(cfg, err, prev, continuity_weight)
        if return_all:
            return best, score, (seeds, cfg, err)
        return best


def sqp_ik_solve_cuda_batch(model, target_links, target_T, previous_cfgs, **kw):
    """Functional form: builds an ``SqpSolver`` and solves."""
    ctor = {k: kw.pop(k) for k in ("spheres", "world", "enable_collision", "collision_weight", "collision_margin",
                                   "device") if k in kw}
    s = SqpSolver(model, target_links, **ctor)
    return s.solve(torch.as_tensor(np.asarray(target_T), device=s.device),
                   torch.as_tensor(np.asarray(previous_cfgs), device=s.device), **kw)
