"""``ls_ik_cuda`` -- drop-in for ``src/pyroffi/cuda_kernels/_ls_ik_cuda.py:76``.

Same arguments (keyword-only solver attributes included) and outputs
``(cfgs[n_problems, n_seeds, n_act], errors[n_problems, n_seeds])`` on torch
CUDA tensors; launches ``pk_ls_ik_cuda`` (reference damping factors x0.5 /
x3) on the current stream.
"""

from __future__ import annotations

import torch

from .. import _lib
from .._tensors import f32, i32, ptr, require_cuda, stream_ptr


def ls_ik_cuda(seeds, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
               topo_inv, target_jnts, ancestor_masks, target_T, robot_spheres_local,
               robot_sphere_joint_idx, world_spheres, world_capsules, world_boxes, world_halfspaces,
               lower, upper, fixed_mask, *, max_iter: int, pos_weight: float, ori_weight: float,
               lambda_init: float, eps_pos: float, eps_ori: float, enable_collision: bool = False,
               collision_weight: float = 0.0, collision_margin: float = 0.02):
    dev = require_cuda(seeds)
    P, Sd, n_act = (int(x) for x in seeds.shape)
    n_joints = int(twists.shape[0])
    n_ee = int(target_jnts.shape[0])
    s = f32(seeds)
    model = [f32(twists), f32(parent_tf), i32(parent_idx), i32(act_idx), f32(mimic_mul),
             f32(mimic_off), i32(mimic_act_idx), i32(topo_inv)]
    rest = [i32(target_jnts), i32(ancestor_masks), f32(target_T), f32(robot_spheres_local),
            i32(robot_sphere_joint_idx), f32(world_spheres), f32(world_capsules), f32(world_boxes),
            f32(world_halfspaces), f32(lower), f32(upper), i32(fixed_mask)]
    model = [t.to(dev) for t in model]
    rest = [t.to(dev) for t in rest]
    out_cfg = torch.empty((P, Sd, n_act), dtype=torch.float32, device=dev)
    out_err = torch.empty((P, Sd), dtype=torch.float32, device=dev)
    n_rs = int(rest[3].shape[0])
    Ms, Mc, Mb, Mh = (int(rest[k].shape[0]) for k in (5, 6, 7, 8))
    _lib.call("pk_ls_ik_cuda", stream_ptr(dev), ptr(s), *[ptr(t) for t in model], *[ptr(t) for t in rest],
              int(max_iter), float(pos_weight), float(ori_weight), float(lambda_init), float(eps_pos),
              float(eps_ori), int(bool(enable_collision)), float(collision_weight),
              float(collision_margin), ptr(out_cfg), ptr(out_err), P, Sd, n_act, n_joints, n_ee, n_rs,
              Ms, Mc, Mb, Mh)
    return out_cfg, out_err
