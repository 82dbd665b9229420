"""Device-resident copies of a robot description, its spheres and a world.

Uploads happen once per object (the caller keeps the ``Device*`` handle);
nothing is cached by raw pointer identity.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .robot import RobotModel, RobotSpheres


def _t(x, dtype, device):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=device)


@dataclass
class DeviceRobot:
    model: RobotModel
    twists: torch.Tensor
    parent_tf: torch.Tensor
    parent_idx: torch.Tensor
    act_idx: torch.Tensor
    mimic_mul: torch.Tensor
    mimic_off: torch.Tensor
    mimic_act_idx: torch.Tensor
    topo_inv: torch.Tensor
    fk_level_starts: torch.Tensor
    fk_level_joints: torch.Tensor
    parent_joint_indices: torch.Tensor
    lower: torch.Tensor
    upper: torch.Tensor

    @classmethod
    def upload(cls, model: RobotModel, device="cuda") -> "DeviceRobot":
        f, i = torch.float32, torch.int32
        return cls(model, _t(model.twists, f, device), _t(model.parent_tf, f, device),
                   _t(model.parent_idx, i, device), _t(model.act_idx, i, device),
                   _t(model.mimic_mul, f, device), _t(model.mimic_off, f, device),
                   _t(model.mimic_act_idx, i, device), _t(model.topo_inv, i, device),
                   _t(model.fk_level_starts, i, device), _t(model.fk_level_joints, i, device),
                   _t(model.parent_joint_indices, i, device), _t(model.lower, f, device),
                   _t(model.upper, f, device))

    def fk_args(self):
        """The 8 model buffers in FFI order (twists .. topo_inv)."""
        return [self.twists, self.parent_tf, self.parent_idx, self.act_idx, self.mimic_mul,
                self.mimic_off, self.mimic_act_idx, self.topo_inv]


@dataclass
class DeviceWorld:
    spheres: torch.Tensor
    capsules: torch.Tensor
    boxes: torch.Tensor
    halfspaces: torch.Tensor

    @classmethod
    def upload(cls, world, device="cuda") -> "DeviceWorld":
        f = torch.float32
        return cls(_t(world.spheres.reshape(-1, 4), f, device), _t(world.capsules.reshape(-1, 7), f, device),
                   _t(world.boxes.reshape(-1, 15), f, device), _t(world.halfspaces.reshape(-1, 6), f, device))

    def arrays(self):
        return [self.spheres, self.capsules, self.boxes, self.halfspaces]

    def counts(self):
        return [int(a.shape[0]) for a in self.arrays()]


@dataclass
class DeviceSpheres:
    link_spheres: torch.Tensor    # [N, S, 4]
    n_links: int
    S: int

    @classmethod
    def upload(cls, spheres: RobotSpheres, device="cuda") -> "DeviceSpheres":
        return cls(_t(spheres.link_spheres(), torch.float32, device), spheres.n_links, spheres.S)
