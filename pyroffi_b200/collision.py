"""Fused FK -> link poses -> sphere world centres -> world distances.

One launch of ``pk_fk_sphere_collision`` replaces the reference chain
``Robot.forward_kinematics`` (``src/pyroffi/_robot.py:66-109``) ->
``RobotCollisionSpherized.at_config`` (``src/pyroffi/collision/_robot_collision.py:744-794``)
-> AoS->SoA transpose (``_cuda_collision.py:405-441``) ->
``collision_world_sphere[_reduced]``; intermediate poses and centres never
leave shared memory.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .device import DeviceRobot, DeviceSpheres, DeviceWorld


@dataclass
class FkCollisionResult:
    min_dist: torch.Tensor | None     # [B]
    link_poses: torch.Tensor | None   # [B, N, 7]
    dist_bkm: torch.Tensor | None     # [B, S*N, M]
    dist_bnm: torch.Tensor | None = None  # [B, N, M]
    sphere_centers: torch.Tensor | None = None  # [B, S*N, 4] world centre + radius


def fk_sphere_collision(robot: DeviceRobot, spheres: DeviceSpheres, world: DeviceWorld,
                        cfg: torch.Tensor, *, min_dist: bool = True, link_poses: bool = True,
                        per_sphere: bool = False, per_link: bool = False, sphere_centers: bool = False,
                        out: FkCollisionResult | None = None) -> FkCollisionResult:
    dev = cfg.device
    c = f32(cfg)
    B = int(c.shape[0])
    N, S = spheres.n_links, spheres.S
    Ms, Mc, Mb, Mh = world.counts()
    M = Ms + Mc + Mb + Mh
    if out is None:
        out = FkCollisionResult(
            torch.empty(B, dtype=torch.float32, device=dev) if min_dist else None,
            torch.empty((B, N, 7), dtype=torch.float32, device=dev) if link_poses else None,
            torch.empty((B, S * N, M), dtype=torch.float32, device=dev) if per_sphere else None,
            torch.empty((B, N, M), dtype=torch.float32, device=dev) if per_link else None,
            torch.empty((B, S * N, 4), dtype=torch.float32, device=dev) if sphere_centers else None)
    _lib.call("pk_fk_sphere_collision", stream_ptr(dev), ptr(c), *[ptr(t) for t in robot.fk_args()],
              ptr(robot.parent_joint_indices), ptr(spheres.link_spheres),
              *[ptr(t) for t in world.arrays()], ptr(out.min_dist), ptr(out.link_poses),
              ptr(out.dist_bkm), ptr(out.dist_bnm), ptr(out.sphere_centers), B, robot.model.n_act, robot.model.n_joints, N, S,
              Ms, Mc, Mb, Mh)
    return out
