"""FP64 forward kinematics -- oracle (test infrastructure only).

Restates, on plain numpy arrays:

* ``JointInfo._map_to_full_joint_space`` / ``get_full_config``
  (``src/pyroffi/_robot_urdf_parser.py:70-128``);
* ``RobotURDFParser._topologically_sort_joints`` (``:162-231``, parent
  dependencies) and ``_compute_fk_depth_schedule`` (``:234-267``);
* ``Robot._forward_kinematics_joints`` (``src/pyroffi/_robot.py:198-263``):
  ``T_pc = parent_tf o exp(twist * q)``, ``T_w[j] = T_w[parent] o T_pc`` walked
  in topological order, returned in original joint order;
* ``Robot._link_poses_from_joint_poses`` (``src/pyroffi/_robot.py:180-196``):
  link pose = pose of its parent joint, identity for the base link;
* the ancestor-mask walk of ``ls_ik_solve_cuda_batch``
  (``src/pyroffi/optimization_engines/_ls_ik.py:1090-1102``).
"""

from __future__ import annotations

import numpy as np

from . import se3


def full_config(cfg, act_idx, mimic_mul, mimic_off, mimic_act_idx):
    """Actuated config [..., n_act] -> full joint values [..., n_joints]."""
    cfg = np.asarray(cfg, dtype=np.float64)
    n_act = cfg.shape[-1]
    padded = np.concatenate([cfg, np.zeros((*cfg.shape[:-1], 1))], axis=-1)
    ref = np.where(np.asarray(mimic_act_idx) == -1, act_idx, mimic_act_idx)
    safe = np.where(ref == -1, n_act, ref)
    return padded[..., safe] * np.asarray(mimic_mul, np.float64) + np.asarray(mimic_off, np.float64)


def topo_sort(parent_idx) -> np.ndarray:
    """Greedy parent-first order: repeatedly take the first unsorted joint
    whose parent joint is already placed (roots first)."""
    parent_idx = [int(p) for p in parent_idx]
    remaining = list(range(len(parent_idx)))
    done: set[int] = set()
    order: list[int] = []
    while remaining:
        for pos, j in enumerate(remaining):
            p = parent_idx[j]
            if p == -1 or p in done:
                order.append(j)
                done.add(j)
                remaining.pop(pos)
                break
        else:
            raise ValueError(f"topological sort failed; remaining joints {remaining}")
    return np.asarray(order, dtype=np.int32)


def fk_depth_schedule(parent_idx, topo_inv):
    """Depth-level schedule: (level_starts[L+1], level_joints[n_j], L)."""
    n = len(topo_inv)
    depth = [0] * n
    for j in topo_inv:
        p = int(parent_idx[int(j)])
        depth[int(j)] = 0 if p == -1 else depth[p] + 1
    max_depth = max(depth) if depth else 0
    starts = [0]
    joints: list[int] = []
    for d in range(max_depth + 1):
        for j in topo_inv:
            if depth[int(j)] == d:
                joints.append(int(j))
        starts.append(len(joints))
    return np.asarray(starts, np.int32), np.asarray(joints, np.int32), max_depth + 1


def fk_joints(cfg, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off,
              mimic_act_idx, topo_inv) -> np.ndarray:
    """World pose of every joint, [..., n_joints, 7] in original joint order."""
    q = full_config(cfg, act_idx, mimic_mul, mimic_off, mimic_act_idx)
    tangents = np.asarray(twists, np.float64) * q[..., None]
    T_pc = se3.compose(np.asarray(parent_tf, np.float64), se3.exp(tangents))
    out = np.zeros_like(T_pc)
    for j in topo_inv:
        j = int(j)
        p = int(parent_idx[j])
        out[..., j, :] = T_pc[..., j, :] if p == -1 else se3.compose(out[..., p, :], T_pc[..., j, :])
    return out


def link_poses(T_joints, parent_joint_indices) -> np.ndarray:
    """Link poses [..., n_links, 7]: parent joint's pose, identity for base links."""
    pji = np.asarray(parent_joint_indices)
    safe = np.where(pji == -1, 0, pji)
    out = T_joints[..., safe, :].copy()
    out[..., pji == -1, :] = se3.identity()
    return out


def forward_kinematics(cfg, model) -> np.ndarray:
    """``Robot.forward_kinematics`` on a model dict -> link poses [..., N, 7]."""
    Tj = fk_joints(cfg, model["twists"], model["parent_tf"], model["parent_idx"],
                   model["act_idx"], model["mimic_mul"], model["mimic_off"],
                   model["mimic_act_idx"], model["topo_inv"])
    return link_poses(Tj, model["parent_joint_indices"])


def ancestor_mask(target_joint: int, parent_idx) -> np.ndarray:
    mask = np.zeros(len(parent_idx), dtype=np.int32)
    j = int(target_joint)
    while j >= 0:
        mask[j] = 1
        j = int(parent_idx[j])
    return mask
