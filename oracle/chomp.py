"""CHOMP optimisation loop -- oracle (test infrastructure only, FP64).

Restates ``_optimize_single_traj`` of
``src/pyroffi/optimization_engines/_chomp_optimization.py:207-330`` for one
trajectory, on the oracle's cost (``oracle.traj``) with the collision
gradient by central finite differences:
gradient clip, pinned endpoints, truncated-CG covariant direction on the
pentadiagonal smoothness metric (``:155-205``), 6-point line search with the
per-step clamp, acceptance on a ``min_cost_improve`` decrease, early stop,
growing collision weight.
"""

from __future__ import annotations

import numpy as np

from . import traj as otraj

ALPHAS = (1.0, 0.5, 0.25, 0.1, 0.05, 0.0)


def metric_apply(x, reg):
    y = 6.0 * x
    y[1:] += -4.0 * x[:-1]
    y[:-1] += -4.0 * x[1:]
    y[2:] += x[:-2]
    y[:-2] += x[2:]
    return y + reg * x


def cg_solve(b, reg, n_iters, tol):
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr = float(r @ r)
    tol2 = (tol * np.sqrt(float(b @ b) + 1e-18) + 1e-12) ** 2
    active = True
    for _ in range(n_iters):
        if not active:
            break
        Ap = metric_apply(p, reg)
        alpha = rr / (float(p @ Ap) + 1e-9)
        x = x + alpha * p
        r = r - alpha * Ap
        rr_new = float(r @ r)
        beta = rr_new / (rr + 1e-9)
        p = r + beta * p
        rr = rr_new
        active = rr_new > tol2
    return x


def chomp_single(init, start, goal, model, link_centers, link_radii, link_pairs, world, lower, upper, cfg):
    """Run cfg.n_iters CHOMP steps on one trajectory [T, n]; returns (traj, history of costs)."""
    x = np.array(init, np.float64)
    x[0], x[-1] = start, goal
    w = cfg.w_collision
    stall, active = 0, True

    def cost(t, wc):
        return otraj.total_cost(t, model, link_centers, link_radii, link_pairs, world, margin=cfg.collision_margin,
                                w_smooth=cfg.w_smooth, w_acc=cfg.w_acc, w_jerk=cfg.w_jerk, w_limits=cfg.w_limits,
                                w_coll=wc, lower=lower, upper=upper)

    hist = []
    for _ in range(cfg.n_iters):
        if not active:
            break
        c = cost(x, w)
        g = (cfg.w_smooth * otraj.smoothness_grad(x, cfg.w_acc, cfg.w_jerk)
             + cfg.w_limits * otraj.limits_grad(x, lower, upper)
             + w * otraj.collision_grad_fd(x, model, link_centers, link_radii, link_pairs, world,
                                           cfg.collision_margin))
        gn = np.linalg.norm(g)
        if cfg.grad_clip_norm > 0 and gn > cfg.grad_clip_norm:
            g = g * (cfg.grad_clip_norm / (gn + 1e-12))
        g[0] = 0.0
        g[-1] = 0.0
        d = np.zeros_like(g)
        if cfg.use_covariant_update and x.shape[0] > 2:
            for k in range(x.shape[1]):
                d[1:-1, k] = -cg_solve(g[1:-1, k].copy(), cfg.smoothness_reg, cfg.n_cg_iters, cfg.cg_tol)
        else:
            d = -g
        trials, tcost = [], []
        for a in ALPHAS:
            t = x + np.clip(a * cfg.step_size * d, -cfg.max_delta_per_step, cfg.max_delta_per_step)
            t[0], t[-1] = start, goal
            trials.append(t)
            tcost.append(cost(t, w))
        i = int(np.argmin(tcost))
        improved = tcost[i] < c - cfg.min_cost_improve
        if improved:
            x = trials[i]
        stall = 0 if improved else stall + 1
        active = stall < cfg.early_stop_patience
        w = min(w * cfg.collision_penalty_scale, cfg.w_collision_max)
        hist.append(c)
    return x, hist
