"""CHOMP trajectory cost with a hand-written adjoint on the GPU.

``TrajectoryCost`` holds a device copy of the robot, its link spheres, the
active self link pairs, the world and the cost weights, and evaluates for a
batch of trajectories ``traj [B, T, n]``:

* ``cost(traj)``           -> J [B]                 (forward only)
* ``grad(traj)``           -> dJ/dtraj [B, T, n]    (backward; link poses recomputed)
* ``cost_and_grad(traj)``  -> both in one launch    (what a CHOMP step needs)

with J = w_smooth * smoothness + w_limits * limits + w_coll * collision as
``cost_fn`` of ``chomp_trajopt``
(``src/pyroffi/optimization_engines/_chomp_optimization.py:243-249``).
``TrajectoryCostFn`` wraps it as a ``torch.autograd.Function``: its forward
runs the cost kernel, its backward re-runs the kernel for the gradient
(recomputing the link transforms instead of storing them) and scales it by
the incoming gradient.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .device import DeviceRobot, DeviceWorld
from .robot import RobotModel, RobotSpheres


class TrajectoryCost:
    def __init__(self, model: RobotModel, spheres: RobotSpheres, world, link_pairs: np.ndarray, *,
                 margin: float = 0.01, w_smooth: float = 1.0, w_acc: float = 0.5, w_jerk: float = 0.1,
                 w_limits: float = 1.0, w_coll: float = 3.0, device="cuda"):
        self.device = torch.device(device)
        self.model = model
        self.robot = DeviceRobot.upload(model, self.device)
        self.world = DeviceWorld.upload(world, self.device)
        self.link_spheres = torch.as_tensor(spheres.link_spheres(), device=self.device)
        self.N, self.S = spheres.n_links, spheres.S
        lp = np.asarray(link_pairs, np.int32).reshape(-1, 2)
        self.pair_i = torch.as_tensor(np.ascontiguousarray(lp[:, 0]), device=self.device)
        self.pair_j = torch.as_tensor(np.ascontiguousarray(lp[:, 1]), device=self.device)
        self.opt = _lib.TrajOptions(margin, w_smooth, w_acc, w_jerk, w_limits, w_coll)

    def _run(self, traj: torch.Tensor, want_cost: bool, want_grad: bool, want_wp: bool = False, active=None):
        """``active`` (optional, uint8/bool [P] on the device): trajectory b is
        evaluated only when active[b % P]; the rows of the others in the
        returned tensors are then left unset (for an optimiser that reads
        only its unfinished trajectories)."""
        x = f32(traj)
        B, T, n = (int(v) for v in x.shape)
        if active is not None:
            self.opt.active, self.opt.active_period = active.data_ptr(), int(active.numel())
        else:
            self.opt.active, self.opt.active_period = None, 0
        cost = torch.empty(B, dtype=torch.float32, device=self.device) if want_cost else None
        grad = torch.empty((B, T, n), dtype=torch.float32, device=self.device) if want_grad else None
        wp = torch.empty((B, T), dtype=torch.float32, device=self.device) if want_wp else None
        r = self.robot
        Ms, Mc, Mb, Mh = self.world.counts()
        _lib.call("pk_traj_cost_grad", stream_ptr(self.device), ctypes.byref(self.opt), ptr(x),
                  *[ptr(t) for t in r.fk_args()], ptr(r.parent_joint_indices), ptr(self.link_spheres),
                  ptr(self.pair_i), ptr(self.pair_j), *[ptr(t) for t in self.world.arrays()], ptr(r.lower),
                  ptr(r.upper), ptr(cost), ptr(grad), ptr(wp), B, T, n, self.model.n_joints, self.N, self.S,
                  int(self.pair_i.shape[0]), Ms, Mc, Mb, Mh)
        return cost, grad, wp

    def cost(self, traj, active=None):
        return self._run(traj, True, False, active=active)[0]

    def grad(self, traj, active=None):
        return self._run(traj, False, True, active=active)[1]

    def cost_and_grad(self, traj, active=None):
        c, g, _ = self._run(traj, True, True, active=active)
        return c, g

    def waypoint_collision(self, traj):
        return self._run(traj, False, False, True)[2]


class TrajectoryCostFn(torch.autograd.Function):
    """J = TrajectoryCostFn.apply(traj, cost_obj) with J [B]; backward gives
    dL/dtraj = dL/dJ[b] * dJ_b/dtraj from the adjoint kernel."""

    @staticmethod
    def forward(ctx, traj, cost_obj: TrajectoryCost):
        ctx.cost_obj = cost_obj
        ctx.save_for_backward(traj)
        return cost_obj.cost(traj.detach())

    @staticmethod
    def backward(ctx, grad_out):
        (traj,) = ctx.saved_tensors
        g = ctx.cost_obj.grad(traj.detach())
        return grad_out.to(g.dtype)[:, None, None] * g, None
