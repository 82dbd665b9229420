"""CHOMP trajectory optimisation on the GPU, driven by the hand-written adjoint.

Restates ``chomp_trajopt`` (``src/pyroffi/optimization_engines/_chomp_optimization.py:155-420``)
for a batch of trajectories at once, with every trajectory's state kept on
the device:

    q_{k+1} = q_k + clip(a * d_k, +-max_delta),   d_k = -M^{-1} clip(grad J(q_k))

* cost and gradient of all B trajectories from one ``pk_traj_cost_grad``
  launch (``TrajectoryCost.cost_and_grad``);
* global-norm gradient clipping per trajectory, pinned endpoints;
* covariant direction: the interior of each joint's timeline is solved
  against the pentadiagonal smoothness metric ``6x - 4(x[t-1] + x[t+1]) +
  (x[t-2] + x[t+2]) + reg x`` by the same truncated conjugate gradient as the
  reference (``n_cg_iters`` steps, relative tolerance ``cg_tol``), batched
  over all (trajectory, joint) timelines, in FP64;
* line search over ``step_size * (1, .5, .25, .1, .05, 0)``: the 6B trial
  trajectories are costed in one more launch, the first minimum wins and is
  taken when it improves the cost by ``min_cost_improve``;
* per-trajectory early stop after ``early_stop_patience`` stalled steps; the
  collision weight grows by ``collision_penalty_scale`` per step up to
  ``w_collision_max``; the final ranking uses ``w_collision_max``.

The iterations have no host round trip, so the whole optimisation is
captured once in a CUDA graph and replayed (``graph=True``).
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

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


def metric_apply(x: torch.Tensor, reg: float) -> torch.Tensor:
    """The interior smoothness metric along dim 1 of x [V, Tin] (zero outside)."""
    y = 6.0 * x + reg * x
    y[:, 1:] -= 4.0 * x[:, :-1]
    y[:, :-1] -= 4.0 * x[:, 1:]
    y[:, 2:] += x[:, :-2]
    y[:, :-2] += x[:, 2:]
    return y


def cg_solve(b: torch.Tensor, reg: float, n_iters: int, tol: float) -> torch.Tensor:
    """Truncated CG for M x = b, one system per row of b [V, Tin]; a row
    stops updating once its squared residual falls below (tol |b| + 1e-12)^2."""
    x = torch.zeros_like(b)
    r = b.clone()
    p = r.clone()
    rr = (r * r).sum(dim=1)
    bnorm = torch.sqrt((b * b).sum(dim=1) + 1e-18)
    tol2 = (tol * bnorm + 1e-12) ** 2
    active = torch.ones_like(rr, dtype=torch.bool)
    for _ in range(n_iters):
        Ap = metric_apply(p, reg)
        alpha = rr / ((p * Ap).sum(dim=1) + 1e-9)
        x_new = x + alpha[:, None] * p
        r_new = r - alpha[:, None] * Ap
        rr_new = (r_new * r_new).sum(dim=1)
        beta = rr_new / (rr + 1e-9)
        p_new = r_new + beta[:, None] * p
        a = active[:, None]
        x = torch.where(a, x_new, x)
        r = torch.where(a, r_new, r)
        p = torch.where(a, p_new, p)
        rr = torch.where(active, rr_new, rr)
        active = active & (rr_new > tol2)
    return x


def _direction(grad: torch.Tensor, cfg: ChompConfig) -> torch.Tensor:
    B, T, n = grad.shape
    if not cfg.use_covariant_update or T <= 2:
        return -grad
    # FP64: truncated CG on this ill-conditioned metric is rounding-sensitive
    # (FP32 runs drift by tens of percent from the FP64 iterates)
    g = grad[:, 1:-1, :].permute(0, 2, 1).reshape(B * n, T - 2).to(torch.float64)
    x = cg_solve(g, cfg.smoothness_reg, cfg.n_cg_iters, cfg.cg_tol)
    d = torch.zeros_like(grad)
    d[:, 1:-1, :] = -x.to(grad.dtype).reshape(B, n, T - 2).permute(0, 2, 1)
    return d


class ChompOptimizer:
    """``run(init_trajs, start, goal)`` -> (best_traj [T, n], costs [B], final_trajs [B, T, n])."""

    def __init__(self, cost: TrajectoryCost, cfg: ChompConfig = ChompConfig()):
        self.cost, self.cfg = cost, cfg
        o = cost.opt
        o.w_smooth, o.w_acc, o.w_jerk, o.w_limits = cfg.w_smooth, cfg.w_acc, cfg.w_jerk, cfg.w_limits
        o.margin = cfg.collision_margin
        self._graph = None

    def _alphas(self, dev):
        # created before any capture: a host-to-device copy cannot be captured
        if getattr(self, "_alpha_t", None) is None or self._alpha_t.device != dev:
            self._alpha_t = torch.tensor(LINE_SEARCH, dtype=torch.float32, device=dev) * self.cfg.step_size
        return self._alpha_t

    def _costs(self, trajs, w_coll, grad=False):
        self.cost.opt.w_coll = float(w_coll)
        return self.cost.cost_and_grad(trajs) if grad else self.cost.cost(trajs)

    def _iterate(self, traj, start, goal):
        cfg = self.cfg
        B = traj.shape[0]
        dev = traj.device
        alphas = self._alphas(dev)
        active = torch.ones(B, dtype=torch.bool, device=dev)
        stall = torch.zeros(B, dtype=torch.int32, device=dev)
        w = cfg.w_collision
        for _ in range(cfg.n_iters):
            c, g = self._costs(traj, w, grad=True)
            if cfg.grad_clip_norm > 0:
                gn = torch.sqrt((g * g).sum(dim=(1, 2)))
                scale = torch.where(gn > cfg.grad_clip_norm, cfg.grad_clip_norm / (gn + 1e-12), torch.ones_like(gn))
                g = g * scale[:, None, None]
            g[:, 0] = 0.0
            g[:, -1] = 0.0
            d = _direction(g, cfg)
            trials = traj[None] + torch.clamp(alphas[:, None, None, None] * d[None], -cfg.max_delta_per_step,
                                              cfg.max_delta_per_step)
            trials[:, :, 0] = start
            trials[:, :, -1] = goal
            tc = self._costs(trials.reshape(-1, *traj.shape[1:]).contiguous(), w).reshape(len(LINE_SEARCH), B)
            best_cost, best_idx = torch.min(tc, dim=0)          # first minimum
            best = trials[best_idx, torch.arange(B, device=dev)]
            improved = best_cost < (c - cfg.min_cost_improve)
            take = active & improved
            traj = torch.where(take[:, None, None], best, traj)
            stall = torch.where(active, torch.where(improved, torch.zeros_like(stall), stall + 1), stall)
            active = active & (stall < cfg.early_stop_patience)
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
