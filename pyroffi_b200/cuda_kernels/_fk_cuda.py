"""``fk_cuda`` -- drop-in for the reference's ``src/pyroffi/cuda_kernels/_fk_cuda.py:52``.

Same arguments and output: world pose of every joint, ``(*batch, n_joints, 7)``
wxyz_xyz, float32.  Tensors are torch CUDA tensors; the call launches
``pk_fk_cuda`` on the current stream.
"""

from __future__ import annotations

import torch

from .. import _lib
from .._tensors import f32, i32, ptr, require_cuda, stream_ptr


def fk_cuda(cfg, twists, parent_tf, parent_idx, act_idx, mimic_mul, mimic_off, mimic_act_idx,
            topo_inv, fk_level_starts, fk_level_joints) -> torch.Tensor:
    dev = require_cuda(cfg)
    batch_axes = tuple(cfg.shape[:-1])
    n_act = int(cfg.shape[-1])
    n_joints = int(twists.shape[0])
    cfg_flat = f32(cfg.reshape(-1, n_act))
    args = [f32(twists), f32(parent_tf), i32(parent_idx), i32(act_idx), f32(mimic_mul),
            f32(mimic_off), i32(mimic_act_idx), i32(topo_inv), i32(fk_level_starts),
            i32(fk_level_joints)]
    args = [a.to(dev) for a in args]
    out = torch.empty((cfg_flat.shape[0], n_joints, 7), dtype=torch.float32, device=dev)
    _lib.call("pk_fk_cuda", stream_ptr(dev), ptr(cfg_flat), *[ptr(a) for a in args], ptr(out),
              cfg_flat.shape[0], n_act, n_joints, int(fk_level_starts.shape[0]) - 1)
    return out.reshape(*batch_axes, n_joints, 7)
