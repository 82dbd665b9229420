"""SCO trajectory optimisation -- FP64 oracle (test infrastructure only).

Restates the reference's SCO loop for one trajectory, in float64:

* group distances (``_collision_dists_reduced``,
  ``src/pyroffi/optimization_engines/_sco_optimization.py:225-255``, and
  ``sco_compute_coll_dists``, ``src/pyroffi/cuda_kernels/_sco_trajopt_cuda_kernel.cu:193-327``):
  group 0 = self (per active link pair, the minimum over all sphere pairs --
  or over equal sphere indices, the JAX self distance), groups 1-4 = world
  spheres / capsules / boxes / halfspaces (per (link, obstacle), the minimum
  over the link's spheres); each group is the smooth minimum
  ``-tau logsumexp(-d / tau)`` of its pair distances, 1e10 without pairs;
* Jacobians by central differences of those (the reference kernel uses
  step 1e-4 in float32; here any step, in float64);
* the inner L-BFGS solve of the convex model (``_lbfgs_inner_solve``,
  ``:296-448``; kernel ``:759-888``): smoothness without a velocity term
  (the kernel ignores ``w_vel``), limits, linearised collision hinge, trust
  region, pinned endpoints, two-loop recursion with Shanno-Kettler scaling,
  5-point line search, best iterate kept;
* the nonlinear ranking cost (``_eval_cost``, ``:455-474``; kernel
  ``:893-1072``);
* the outer loop with penalty continuation (``_sco_trajopt_jax``, ``:481-502``).

Link poses are the poses of the links' parent joints (the robot's FK).
Parity is pinned through the shared primitives (FK, sphere-to-primitive
distances, ``colldist_from_sdf``), which are checked against the
reference's golden vectors; the SCO loop itself has no reference output to
pin against here (the reference kernel needs JAX / XLA FFI to run).
"""

from __future__ import annotations

import numpy as np

from . import collision, kinematics

ACC_STENCIL = np.array([-1.0, 16.0, -30.0, 16.0, -1.0]) / 12.0
LS_ALPHAS = (1.0, 0.5, 0.25, 0.1, 0.025)
N_GROUPS = 5


def link_spheres_world(cfgs, model, link_centers, link_radii):
    """cfgs [C, n] -> centres [C, N, S, 3], radii [N, S] (link pose = parent joint pose)."""
    Tj = kinematics.fk_joints(np.asarray(cfgs, np.float64), model["twists"], model["parent_tf"],
                              model["parent_idx"], model["act_idx"], model["mimic_mul"], model["mimic_off"],
                              model["mimic_act_idx"], model["topo_inv"])
    links = kinematics.link_poses(Tj, model["parent_joint_indices"])          # [C, N, 7]
    cen = collision.transform_points(links[:, :, None, :], np.asarray(link_centers, np.float64)[None])
    return cen, np.asarray(link_radii, np.float64)


def pair_distances(cfgs, model, link_centers, link_radii, link_pairs, world, self_all=True):
    """Per configuration the pair distances of each group: a list (length C) of
    5 arrays (self pairs, then (link, obstacle) pairs of each world type)."""
    cen, rad = link_spheres_world(cfgs, model, link_centers, link_radii)
    C, N, S, _ = cen.shape
    valid = rad >= 0
    has = valid.any(axis=1)
    lp = np.asarray(link_pairs, np.int64).reshape(-1, 2)
    ws, wc, wb, wh = (np.asarray(a, np.float64).reshape(-1, k) for a, k in zip(world, (4, 7, 15, 6)))
    out = []
    for c in range(C):
        groups = []
        sd = []
        for li, lj in lp:
            if li == lj or not (0 <= li < N and 0 <= lj < N) or not has[li] or not has[lj]:
                continue
            a, b = cen[c, li], cen[c, lj]
            d = np.linalg.norm(a[:, None, :] - b[None, :, :], axis=-1) - (rad[li][:, None] + rad[lj][None, :])
            m = valid[li][:, None] & valid[lj][None, :]
            if not self_all:
                m = m & np.eye(S, dtype=bool)
            if m.any():
                sd.append(d[m].min())
        groups.append(np.array(sd))
        for k, arr in enumerate((ws, wc, wb, wh)):
            vals = []
            for l in range(N):
                if not has[l] or len(arr) == 0:
                    continue
                p, r = cen[c, l][valid[l]], rad[l][valid[l]]
                pe, re = p[:, None, :], r[:, None]
                if k == 0:
                    d = collision.sphere_sphere(pe, re, arr[:, :3], arr[:, 3])
                elif k == 1:
                    d = collision.sphere_capsule(pe, re, arr[:, 0:3], arr[:, 3:6], arr[:, 6])
                elif k == 2:
                    d = collision.sphere_box(pe, re, arr)
                else:
                    d = collision.sphere_halfspace(pe, re, arr)
                vals.append(d.min(axis=0))                                      # [M_k]
            groups.append(np.concatenate(vals) if vals else np.zeros(0))
        out.append(groups)
    return out


def smooth_min(d, tau):
    d = np.asarray(d, np.float64)
    if d.size == 0:
        return 1e10
    e = -d / tau
    m = e.max()
    return -tau * (np.log(np.exp(e - m).sum()) + m)


def group_dists(cfgs, model, link_centers, link_radii, link_pairs, world, tau, self_all=True):
    """[C, 5] smooth-min distances."""
    pd = pair_distances(cfgs, model, link_centers, link_radii, link_pairs, world, self_all)
    return np.array([[smooth_min(g, tau) for g in groups] for groups in pd])


def group_jacobian(cfgs, model, link_centers, link_radii, link_pairs, world, tau, self_all=True, eps=1e-6):
    """[C, 5, n] central differences of ``group_dists``."""
    q = np.asarray(cfgs, np.float64)
    C, n = q.shape
    rows = [q]
    for d in range(n):
        e = np.zeros(n)
        e[d] = eps
        rows += [q + e, q - e]
    allq = np.concatenate(rows, axis=0)
    g = group_dists(allq, model, link_centers, link_radii, link_pairs, world, tau, self_all)
    J = np.zeros((C, N_GROUPS, n))
    for d in range(n):
        J[:, :, d] = (g[C * (1 + 2 * d):C * (2 + 2 * d)] - g[C * (2 + 2 * d):C * (3 + 2 * d)]) / (2.0 * eps)
    return J


def coll_sum(cfgs, model, link_centers, link_radii, link_pairs, world, margin, self_all=True):
    """[C] sum of -colldist_from_sdf over every pair distance (ranking cost's collision part)."""
    pd = pair_distances(cfgs, model, link_centers, link_radii, link_pairs, world, self_all)
    return np.array([sum(float(-collision.colldist_from_sdf(g, margin).sum()) for g in groups) for groups in pd])


# ---------------------------------------------------------------------------
# convex model and inner L-BFGS
# ---------------------------------------------------------------------------

def _acc(x):
    T = x.shape[0]
    if T < 5:
        return np.zeros((0, x.shape[1]))
    return sum(ACC_STENCIL[i] * x[i:T - 4 + i] for i in range(5))


def smoothness(x, w_acc, w_jerk):
    a = _acc(x)
    j = a[1:] - a[:-1]
    return w_acc * np.sum(a ** 2) + w_jerk * np.sum(j ** 2)


def smoothness_grad(x, w_acc, w_jerk):
    T = x.shape[0]
    a = _acc(x)
    g = np.zeros_like(x)
    if a.shape[0] == 0:
        return g
    j = a[1:] - a[:-1]
    ga = 2.0 * w_acc * a
    ga[1:] += 2.0 * w_jerk * j
    ga[:-1] -= 2.0 * w_jerk * j
    for i in range(5):
        g[i:T - 4 + i] += ACC_STENCIL[i] * ga
    return g


def model_cost(x, qk, dk, Jk, lower, upper, cfg, w_coll):
    """Convex model of the inner solve (x, qk [T, n]; dk [T, 5]; Jk [T, 5, n])."""
    delta = x - qk
    dl = dk + np.einsum("tgd,td->tg", Jk, delta)
    v = np.maximum(0.0, cfg.collision_margin - dl)
    lim = np.maximum(0.0, x - upper) + np.maximum(0.0, lower - x)
    return (cfg.w_smooth * smoothness(x, cfg.w_acc, cfg.w_jerk) + cfg.w_limits * np.sum(lim ** 2)
            + w_coll * np.sum(v ** 2) + cfg.w_trust * np.sum(delta ** 2))


def model_grad(x, qk, dk, Jk, lower, upper, cfg, w_coll):
    delta = x - qk
    dl = dk + np.einsum("tgd,td->tg", Jk, delta)
    v = np.maximum(0.0, cfg.collision_margin - dl)
    g = cfg.w_smooth * smoothness_grad(x, cfg.w_acc, cfg.w_jerk)
    g += 2.0 * cfg.w_limits * (np.maximum(0.0, x - upper) - np.maximum(0.0, lower - x))
    g += np.einsum("tg,tgd->td", -2.0 * w_coll * v, Jk)
    g += 2.0 * cfg.w_trust * delta
    g[0] = 0.0
    g[-1] = 0.0
    return g


def lbfgs_inner(qk, dk, Jk, lower, upper, cfg, w_coll):
    """Best iterate of ``n_inner_iters`` L-BFGS steps from x = qk."""
    x = np.array(qk, np.float64)
    qk = np.array(qk, np.float64)
    m = cfg.m_lbfgs
    Sb, Yb = [None] * m, [None] * m
    rho = np.zeros(m)
    m_used, newest = 0, 0
    f = lambda z: model_cost(z, qk, dk, Jk, lower, upper, cfg, w_coll)  # noqa: E731
    cost = f(x)
    g = model_grad(x, qk, dk, Jk, lower, upper, cfg, w_coll)
    best_x, best_cost = x.copy(), cost
    step = np.zeros_like(x)
    g_prev = g.copy()
    for it in range(cfg.n_inner_iters):
        if it > 0:
            cost = f(x)
            g = model_grad(x, qk, dk, Jk, lower, upper, cfg, w_coll)
            y = g - g_prev
            sy, yy = float(np.sum(step * y)), float(np.sum(y * y))
            if sy > 1e-10 * yy + 1e-30:
                newest = (newest + 1) % m
                Sb[newest], Yb[newest], rho[newest] = step.copy(), y, 1.0 / (sy + 1e-30)
                m_used = min(m_used + 1, m)
        g_prev = g.copy()
        if m_used == 0:
            p = -g / (np.sqrt(np.sum(g * g)) + 1e-18)
        else:
            q = g.copy()
            al = np.zeros(m)
            for k in range(m_used):
                i = (newest - k) % m
                al[k] = rho[i] * np.sum(Sb[i] * q)
                q = q - al[k] * Yb[i]
            q = q * (np.sum(Sb[newest] * Yb[newest]) / (np.sum(Yb[newest] * Yb[newest]) + 1e-18))
            for k in range(m_used - 1, -1, -1):
                i = (newest - k) % m
                beta = rho[i] * np.sum(Yb[i] * q)
                q = q + Sb[i] * (al[k] - beta)
            p = -q
        p[0] = 0.0
        p[-1] = 0.0
        tc = [f(x + a * p) for a in LS_ALPHAS]
        best = int(np.argmin(tc))
        for i, c in enumerate(tc):
            if c < cost * (1.0 - 1e-4):
                best = i
                break
        step = LS_ALPHAS[best] * p
        x = x + step
        if tc[best] < best_cost:
            best_x, best_cost = x.copy(), tc[best]
    return best_x


def ranking_cost(traj, model, link_centers, link_radii, link_pairs, world, lower, upper, cfg, self_all=True):
    x = np.asarray(traj, np.float64)
    lim = np.maximum(0.0, x - upper) + np.maximum(0.0, lower - x)
    coll = coll_sum(x, model, link_centers, link_radii, link_pairs, world, cfg.collision_margin, self_all)
    return (cfg.w_smooth * smoothness(x, cfg.w_acc, cfg.w_jerk) + cfg.w_limits * np.sum(lim ** 2)
            + cfg.w_collision_max * float(coll.sum()))


def sco_single(init, start, goal, model, link_centers, link_radii, link_pairs, world, lower, upper, cfg,
               self_all=True, eps=1e-6):
    """Outer loop for one trajectory -> (traj [T, n], ranking cost)."""
    x = np.array(init, np.float64)
    x[0], x[-1] = start, goal
    w = cfg.w_collision
    tau = cfg.smooth_min_temperature
    for _ in range(cfg.n_outer_iters):
        dk = group_dists(x, model, link_centers, link_radii, link_pairs, world, tau, self_all)
        Jk = group_jacobian(x, model, link_centers, link_radii, link_pairs, world, tau, self_all, eps)
        x = lbfgs_inner(x, dk, Jk, lower, upper, cfg, w)
        x[0], x[-1] = start, goal
        w = min(w * cfg.penalty_scale, cfg.w_collision_max)
    return x, ranking_cost(x, model, link_centers, link_radii, link_pairs, world, lower, upper, cfg, self_all)
