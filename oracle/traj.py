"""CHOMP trajectory cost and its gradient -- oracle (test infrastructure only).

Restates ``cost_fn`` of ``chomp_trajopt``
(``src/pyroffi/optimization_engines/_chomp_optimization.py:243-249``) for one
trajectory ``traj [T, n]``:

    J = w_smooth * smoothness + w_limits * limits + w_coll * collision

* ``_smoothness_cost`` (``:93-110``): acc_k = (-x_k + 16 x_{k+1} - 30 x_{k+2}
  + 16 x_{k+3} - x_{k+4}) / 12, jerk_k = acc_{k+1} - acc_k,
  cost = w_acc sum acc^2 + w_jerk sum jerk^2;
* ``_limits_cost`` (``:113-121``): sum (max(0, x - upper) + max(0, lower - x))^2;
* ``_collision_cost`` (``:140-153``): per waypoint, sum over the active self
  link pairs (min over the same sphere index s, ``_robot_collision.py:796-828``)
  and over every (link, obstacle) (min over the link's spheres,
  ``:830-895``) of max(0, margin - d)^2.

Distances follow the CUDA convention (exact norms; the JAX sphere distance
adds 1e-6 to every component before the norm, a <= 1.8e-6 m shift).  The
gradient of the smoothness and limit terms is analytic; the collision
gradient is taken by central finite differences of the FP64 cost (the
reference differentiates it with ``jax.value_and_grad``).
"""

from __future__ import annotations

import numpy as np

from . import collision, kinematics

ACC_STENCIL = np.array([-1.0, 16.0, -30.0, 16.0, -1.0]) / 12.0


def smoothness(traj, w_acc, w_jerk):
    x = np.asarray(traj, np.float64)
    acc = sum(ACC_STENCIL[i] * x[i:x.shape[0] - 4 + i] for i in range(5))
    jerk = acc[1:] - acc[:-1]
    return w_acc * np.sum(acc ** 2) + w_jerk * np.sum(jerk ** 2)


def smoothness_grad(traj, w_acc, w_jerk):
    x = np.asarray(traj, np.float64)
    T = x.shape[0]
    acc = sum(ACC_STENCIL[i] * x[i:T - 4 + i] for i in range(5))
    jerk = acc[1:] - acc[:-1]
    g_acc = 2.0 * w_acc * acc
    g_acc[1:] += 2.0 * w_jerk * jerk
    g_acc[:-1] -= 2.0 * w_jerk * jerk
    g = np.zeros_like(x)
    for i in range(5):
        g[i:T - 4 + i] += ACC_STENCIL[i] * g_acc
    return g


def limits(traj, lower, upper):
    x = np.asarray(traj, np.float64)
    v = np.maximum(0.0, x - upper) + np.maximum(0.0, lower - x)
    return np.sum(v ** 2)


def limits_grad(traj, lower, upper):
    x = np.asarray(traj, np.float64)
    return 2.0 * np.maximum(0.0, x - upper) - 2.0 * np.maximum(0.0, lower - x)


def collision_cost(traj, model, link_centers, link_radii, link_pairs, world, margin):
    """Sum over waypoints of the CHOMP collision hinge (FP64)."""
    Tj = kinematics.fk_joints(traj, model["twists"], model["parent_tf"], model["parent_idx"],
                              model["act_idx"], model["mimic_mul"], model["mimic_off"],
                              model["mimic_act_idx"], model["topo_inv"])
    links = kinematics.link_poses(Tj, model["parent_joint_indices"])
    lp = np.asarray(link_pairs).reshape(-1, 2)
    ws, wc, wb, wh = (np.asarray(a, np.float64) for a in world)
    c = collision.chomp_collision_cost(links, np.asarray(link_centers, np.float64),
                                       np.asarray(link_radii, np.float64), lp[:, 0], lp[:, 1],
                                       ws, wc, wb, wh, margin)
    return float(np.sum(c))


def total_cost(traj, model, link_centers, link_radii, link_pairs, world, *, margin, w_smooth, w_acc,
               w_jerk, w_limits, w_coll, lower, upper):
    return (w_smooth * smoothness(traj, w_acc, w_jerk) + w_limits * limits(traj, lower, upper)
            + w_coll * collision_cost(traj, model, link_centers, link_radii, link_pairs, world, margin))


def collision_grad_fd(traj, model, link_centers, link_radii, link_pairs, world, margin, h=1e-6):
    """Central finite differences of the FP64 collision cost."""
    x = np.array(traj, np.float64)
    g = np.zeros_like(x)
    for t in range(x.shape[0]):
        for d in range(x.shape[1]):
            xp = x.copy()
            xm = x.copy()
            xp[t, d] += h
            xm[t, d] -= h
            # only waypoint t changes: evaluate it alone
            cp = collision_cost(xp[t:t + 1], model, link_centers, link_radii, link_pairs, world, margin)
            cm = collision_cost(xm[t:t + 1], model, link_centers, link_radii, link_pairs, world, margin)
            g[t, d] = (cp - cm) / (2.0 * h)
    return g
