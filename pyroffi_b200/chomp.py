"""CHOMP trajectory optimisation on the GPU, driven by the hand-written adjoint.

Restates ``chomp_trajopt`` (``src/pyroffi/optimization_engines/_chomp_optimization.py:155-420``)
for a batch of trajectories at once, with every trajectory's state kept on
the device:

    q_{k+1} = q_k + clip(a * d_k, +-max_delta),   d_k = -M^{-1} clip(grad J(q_k))

* cost and gradient of all B trajectories from one ``pk_traj_cost_grad``
  launch (``TrajectoryCost.cost_and_grad``);
* global-norm gradient clipping per trajectory, pinned endpoints, and the
  covariant direction -- the interior of each joint's timeline solved
  against the pentadiagonal smoothness metric ``6x - 4(x[t-1] + x[t+1]) +
  (x[t-2] + x[t+2]) + reg x`` by the same truncated conjugate gradient as the
  reference (``n_cg_iters`` steps, relative tolerance ``cg_tol``) in FP64 --
  in one ``pk_chomp_direction`` launch (a warp per (trajectory, joint)
  timeline);
* line search over ``step_size * (1, .5, .25, .1, .05, 0)``: the 5B trial
  trajectories of the non-zero steps are built by ``pk_chomp_line_trials``
  and costed in one more launch (the zero step's trial is the current
  trajectory, costed by the gradient launch); ``pk_chomp_line_select`` takes
  the first minimum when it improves the cost by ``min_cost_improve`` and
  updates the stall counters, in place;
* per-trajectory early stop after ``early_stop_patience`` stalled steps; the
  collision weight grows by ``collision_penalty_scale`` per step up to
  ``w_collision_max``; the final ranking uses ``w_collision_max``.

The iterations have no host round trip, so the whole optimisation is
captured once in a CUDA graph and replayed (``graph=True``).
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .trajopt import TrajectoryCost


@dataclass(frozen=True)
class ChompConfig:
    """Hyper-parameters, with the reference's names and defaults (``ChompTrajOptConfig``)."""
    n_iters: int = 100
    step_size: float = 0.05
    w_smooth: float = 1.0
    w_acc: float = 0.5
    w_jerk: float = 0.1
    w_collision: float = 3.0
    w_collision_max: float = 50.0
    collision_penalty_scale: float = 1.05
    collision_margin: float = 0.01
    w_limits: float = 1.0
    use_covariant_update: bool = True
    smoothness_reg: float = 1e-3
    n_cg_iters: int = 24
    cg_tol: float = 1e-4
    grad_clip_norm: float = 10.0
    max_delta_per_step: float = 0.05
    early_stop_patience: int = 15
    min_cost_improve: float = 1e-5


LINE_SEARCH = (1.0, 0.5, 0.25, 0.1, 0.05, 0.0)


def covariant_direction(grad: torch.Tensor, cfg: ChompConfig, active=None) -> torch.Tensor:
    """Clipped, endpoint-pinned descent direction [B, T, n]: -M^-1 g on each
    joint's interior timeline by the truncated FP64 CG, or -g without the
    covariant update (one ``pk_chomp_direction`` launch).  With ``active``
    (uint8/bool [B] on the device), only those trajectories' rows are set."""
    g = f32(grad)
    B, T, n = (int(v) for v in g.shape)
    d = torch.empty_like(g)
    _lib.call("pk_chomp_direction", stream_ptr(g.device), ptr(g), ptr(d), B, T, n, int(cfg.n_cg_iters),
              float(cfg.grad_clip_norm), float(cfg.smoothness_reg), float(cfg.cg_tol),
              int(bool(cfg.use_covariant_update)), ptr(active))
    return d


class ChompOptimizer:
    """``run(init_trajs, start, goal)`` -> (best_traj [T, n], costs [B], final_trajs [B, T, n]).

    skip_finished: a trajectory that has early-stopped no longer changes, so
    its cost, gradient, direction and line-search trials are skipped from
    then on (the kernels take the ``active`` mask); the results are the same
    bits as without the skip."""

    def __init__(self, cost: TrajectoryCost, cfg: ChompConfig = ChompConfig(), skip_finished: bool = True):
        self.cost, self.cfg = cost, cfg
        self.skip_finished = skip_finished
        o = cost.opt
        o.w_smooth, o.w_acc, o.w_jerk, o.w_limits = cfg.w_smooth, cfg.w_acc, cfg.w_jerk, cfg.w_limits
        o.margin = cfg.collision_margin
        self._graph = None

    def _alphas(self, dev):
        # created before any capture: a host-to-device copy cannot be captured
        if getattr(self, "_alpha_t", None) is None or self._alpha_t.device != dev:
            self._alpha_t = torch.tensor(LINE_SEARCH, dtype=torch.float32, device=dev) * self.cfg.step_size
        return self._alpha_t

    def _costs(self, trajs, w_coll, grad=False, active=None):
        self.cost.opt.w_coll = float(w_coll)
        return self.cost.cost_and_grad(trajs, active) if grad else self.cost.cost(trajs, active)

    def _iterate(self, traj, start, goal):
        cfg = self.cfg
        B = traj.shape[0]
        dev = traj.device
        alphas = self._alphas(dev)
        start, goal = f32(start), f32(goal)
        active = torch.ones(B, dtype=torch.bool, device=dev)
        stall = torch.zeros(B, dtype=torch.int32, device=dev)
        w = cfg.w_collision
        traj = traj.contiguous()
        K = len(LINE_SEARCH) - 1
        T, n = int(traj.shape[1]), int(traj.shape[2])
        trials = torch.empty((K, B, T, n), dtype=torch.float32, device=dev)
        st = stream_ptr(dev)
        # finished (early-stopped) trajectories are skipped: the selection reads nothing of theirs
        act = active if self.skip_finished else None
        for _ in range(cfg.n_iters):
            c, g = self._costs(traj, w, grad=True, active=act)
            d = covariant_direction(g, cfg, act)
            # the last trial step is 0: that trial is the current trajectory, whose cost
            # the gradient launch has just produced, so only the K others are built and costed
            _lib.call("pk_chomp_line_trials", st, ptr(traj), ptr(d), ptr(alphas), K, float(cfg.max_delta_per_step),
                      ptr(start), ptr(goal), ptr(trials), B, T, n, ptr(act))
            tc = self._costs(trials.view(K * B, T, n), w, active=act)
            # first minimum over the trials and the current cost; step, stall count, early stop (in place)
            _lib.call("pk_chomp_line_select", st, ptr(tc), ptr(c), ptr(trials), ptr(traj), ptr(active), ptr(stall), K,
                      float(cfg.min_cost_improve), int(cfg.early_stop_patience), B, T, n)
            w = min(w * cfg.collision_penalty_scale, cfg.w_collision_max)
        final_costs = self._costs(traj, cfg.w_collision_max)
        return traj, final_costs

    def run(self, init_trajs: torch.Tensor, start: torch.Tensor, goal: torch.Tensor, graph: bool = False):
        traj = init_trajs.to(torch.float32).clone()
        traj[:, 0] = start
        traj[:, -1] = goal
        if not graph:
            final, costs = self._iterate(traj, start, goal)
        else:
            if self._graph is None or self._g_in.shape != traj.shape:
                self._g_in = traj.clone()
                self._g_start, self._g_goal = start.clone(), goal.clone()
                torch.cuda.synchronize()
                s = torch.cuda.Stream()
                s.wait_stream(torch.cuda.current_stream())
                with torch.cuda.stream(s):
                    self._iterate(self._g_in.clone(), self._g_start, self._g_goal)  # warm-up outside capture
                torch.cuda.current_stream().wait_stream(s)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, capture_error_mode="relaxed"):
                    self._g_out = self._iterate(self._g_in.clone(), self._g_start, self._g_goal)
                self._graph = g
            self._g_in.copy_(traj)
            self._g_start.copy_(start)
            self._g_goal.copy_(goal)
            self._graph.replay()
            final, costs = self._g_out
        return final[int(torch.argmin(costs))], costs, final


def chomp_trajopt(init_trajs, start, goal, cost: TrajectoryCost, cfg: ChompConfig = ChompConfig(), graph=False):
    """Functional form of ``chomp_trajopt(..., use_cuda=True)``."""
    return ChompOptimizer(cost, cfg).run(init_trajs, start, goal, graph=graph)
