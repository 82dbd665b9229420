"""SCO trajectory optimisation on the GPU (sequential convex optimisation).

Drop-in for ``sco_trajopt(init_trajs, start, goal, robot, robot_coll,
world_geoms, opt_cfg, use_cuda=True)``
(``src/pyroffi/optimization_engines/_sco_optimization.py:505-551``): every
outer iteration linearises the collision distances of all waypoints of all
trajectories at once (five smooth-min groups: self, world spheres, capsules,
boxes, halfspaces, each with its Jacobian), solves the convex subproblem of
each trajectory by L-BFGS, and raises the collision weight; the trajectories
are finally ranked by their nonlinear cost at ``w_collision_max``.

* ``ScoOptimizer.run`` is one call of ``pk_sco_trajopt`` (the whole loop on
  the stream; nothing allocates inside, so it can be captured in a CUDA
  graph with ``graph=True``);
* ``linearize``, ``inner`` and ``final_cost`` expose the three stages
  (``pk_sco_linearize``, ``pk_sco_inner``, ``pk_sco_final_cost``);
* ``linearize_fd`` is the reference kernel's central-difference Jacobian
  assembled from distance-only launches.

Conventions: the link pose is the pose of the link's parent joint (the
robot's FK; the reference kernel reads joint poses by link index instead),
the smoothness term has no velocity part (the reference kernel ignores
``w_vel``, as its config documents), and a self pair's distance is the
minimum over all sphere pairs (``self_all_pairs=False``: over equal sphere
indices, the JAX self distance).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._tensors import f32, ptr, stream_ptr
from .device import DeviceRobot, DeviceWorld
from .robot import RobotModel, RobotSpheres

N_GROUPS = 5


@dataclass(frozen=True)
class ScoConfig:
    """Hyper-parameters with the reference's names and defaults (``ScoTrajOptConfig``)."""
    n_outer_iters: int = 10
    n_inner_iters: int = 30
    m_lbfgs: int = 6
    w_smooth: float = 1.0
    w_vel: float = 1.0            # unused, as in the reference kernel
    w_acc: float = 0.5
    w_jerk: float = 0.1
    w_collision: float = 1.0
    w_collision_max: float = 100.0
    penalty_scale: float = 3.0
    collision_margin: float = 0.01
    w_trust: float = 0.5
    w_limits: float = 1.0
    smooth_min_temperature: float = 0.05


class ScoOptimizer:
    def __init__(self, model: RobotModel, spheres: RobotSpheres, world, link_pairs, cfg: ScoConfig = ScoConfig(),
                 *, fd_eps: float = 0.0, self_all_pairs: bool = True, inner_threads: int = 0, device="cuda"):
        self.device = torch.device(device)
        self.model, self.cfg = model, cfg
        self.robot = DeviceRobot.upload(model, self.device)
        self.world = DeviceWorld.upload(world, self.device)
        self.link_spheres = torch.as_tensor(spheres.link_spheres(), device=self.device)
        self.N, self.S = spheres.n_links, spheres.S
        lp = np.asarray(link_pairs, np.int32).reshape(-1, 2)
        if len(lp) and np.any(lp[:, 0] == lp[:, 1]):
            raise ValueError("a self pair must join two different links")
        self.pair_i = torch.as_tensor(np.ascontiguousarray(lp[:, 0]), device=self.device)
        self.pair_j = torch.as_tensor(np.ascontiguousarray(lp[:, 1]), device=self.device)
        self.opt = _lib.ScoOptions(cfg.n_outer_iters, cfg.n_inner_iters, cfg.m_lbfgs, cfg.w_smooth, cfg.w_acc,
                                   cfg.w_jerk, cfg.w_limits, cfg.w_trust, cfg.w_collision, cfg.w_collision_max,
                                   cfg.penalty_scale, cfg.collision_margin, cfg.smooth_min_temperature,
                                   float(fd_eps), int(bool(self_all_pairs)), int(inner_threads))
        self._ws = None
        self._graph = None

    # -- stages -------------------------------------------------------------
    def _robot_args(self):
        r = self.robot
        return [*[ptr(t) for t in r.fk_args()], ptr(r.parent_joint_indices), ptr(self.link_spheres),
                ptr(self.pair_i), ptr(self.pair_j), *[ptr(t) for t in self.world.arrays()]]

    def _extents(self):
        return [self.model.n_joints, self.N, self.S, int(self.pair_i.shape[0]), *self.world.counts()]

    def linearize(self, cfgs: torch.Tensor, *, want_dist=True, want_jac=True, want_coll=False):
        """cfgs [..., n] -> (d [..., 5], J [..., 5, n], coll [...]) (None where not requested)."""
        x = f32(cfgs)
        lead, n = x.shape[:-1], int(x.shape[-1])
        Cn = int(np.prod(lead)) if len(lead) else 1
        d = torch.empty((*lead, N_GROUPS), dtype=torch.float32, device=self.device) if want_dist else None
        J = torch.empty((*lead, N_GROUPS, n), dtype=torch.float32, device=self.device) if want_jac else None
        c = torch.empty(lead, dtype=torch.float32, device=self.device) if want_coll else None
        _lib.call("pk_sco_linearize", stream_ptr(self.device), ctypes.byref(self.opt), ptr(x), *self._robot_args(),
                  ptr(d), ptr(J), ptr(c), Cn, n, *self._extents())
        return d, J, c

    def linearize_fd(self, cfgs: torch.Tensor, eps: float = 1e-4):
        """Central differences of the group distances (the reference kernel's Jacobian)."""
        x = f32(cfgs)
        lead, n = x.shape[:-1], int(x.shape[-1])
        base = x.reshape(-1, n)
        e = torch.eye(n, dtype=torch.float32, device=self.device) * eps
        pert = torch.empty((base.shape[0], 2 * n + 1, n), dtype=torch.float32, device=self.device)
        pert[:, 0] = base
        pert[:, 1::2] = base[:, None, :] + e[None]     # row 2d + 1: +eps on coordinate d
        pert[:, 2::2] = base[:, None, :] - e[None]     # row 2d + 2: -eps
        d, _, _ = self.linearize(pert, want_jac=False)
        d0 = d[:, 0]
        J = (d[:, 1::2] - d[:, 2::2]) * (1.0 / (2.0 * eps))                     # [C, n, 5]
        return d0.reshape(*lead, N_GROUPS), J.transpose(1, 2).reshape(*lead, N_GROUPS, n)

    def inner(self, traj: torch.Tensor, d: torch.Tensor, J: torch.Tensor, w_coll: float, start, goal):
        """One inner solve of every trajectory from its linearisation (returns a new tensor)."""
        x = f32(traj).clone()
        B, T, n = (int(v) for v in x.shape)
        # L-BFGS history buffer, used when the history does not fit in shared memory
        hist = torch.empty(max(1, B * 2 * self.cfg.m_lbfgs * T * n), dtype=torch.float32, device=self.device)
        _lib.call("pk_sco_inner", stream_ptr(self.device), ctypes.byref(self.opt), ptr(x), ptr(f32(d)),
                  ptr(f32(J)), ptr(self.robot.lower), ptr(self.robot.upper), ptr(f32(start)), ptr(f32(goal)),
                  ptr(hist), float(w_coll), B, T, n)
        return x

    def final_cost(self, traj: torch.Tensor):
        x = f32(traj)
        B, T, n = (int(v) for v in x.shape)
        _, _, coll = self.linearize(x, want_dist=False, want_jac=False, want_coll=True)
        cost = torch.empty(B, dtype=torch.float32, device=self.device)
        _lib.call("pk_sco_final_cost", stream_ptr(self.device), ctypes.byref(self.opt), ptr(x), ptr(coll),
                  ptr(self.robot.lower), ptr(self.robot.upper), ptr(cost), B, T, n)
        return cost

    def run_stages(self, init_trajs, start, goal):
        """The loop through the three stage calls (same result as ``run``)."""
        cfg = self.cfg
        x = f32(init_trajs).clone()
        x[:, 0] = f32(start)
        x[:, -1] = f32(goal)
        w = cfg.w_collision
        for _ in range(cfg.n_outer_iters):
            if self.opt.fd_eps > 0:
                d, J = self.linearize_fd(x, self.opt.fd_eps)
            else:
                d, J, _ = self.linearize(x)
            x = self.inner(x, d, J, w, start, goal)
            w = min(w * cfg.penalty_scale, cfg.w_collision_max)
        costs = self.final_cost(x)
        return x[int(torch.argmin(costs))], costs, x

    # -- whole loop -----------------------------------------------------------
    def _workspace(self, B, T, n):
        nb = ctypes.c_size_t(0)
        _lib.call("pk_sco_workspace_bytes", ctypes.byref(self.opt), B, T, n, ctypes.byref(nb))
        need = max(256, int(nb.value))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(need, dtype=torch.uint8, device=self.device)
        return self._ws

    def _call(self, init, start, goal, out, costs):
        B, T, n = (int(v) for v in init.shape)
        ws = self._workspace(B, T, n)
        _lib.call("pk_sco_trajopt", stream_ptr(self.device), ctypes.byref(self.opt), ptr(init), ptr(start),
                  ptr(goal), *self._robot_args(), ptr(self.robot.lower), ptr(self.robot.upper), ptr(out), ptr(costs), ptr(ws),
                  int(ws.numel()), B, T, n, *self._extents())

    def run(self, init_trajs: torch.Tensor, start: torch.Tensor, goal: torch.Tensor, graph: bool = False):
        """-> (best_traj [T, n], costs [B], final_trajs [B, T, n])."""
        init = f32(init_trajs)
        st, gl = f32(start), f32(goal)
        B, T, n = (int(v) for v in init.shape)
        if not graph:
            out = torch.empty_like(init)
            costs = torch.empty(B, dtype=torch.float32, device=self.device)
            self._call(init, st, gl, out, costs)
        else:
            if self._graph is None or self._g_in.shape != init.shape:
                self._g_in, self._g_st, self._g_gl = init.clone(), st.clone(), gl.clone()
                self._g_out = torch.empty_like(init)
                self._g_cost = torch.empty(B, dtype=torch.float32, device=self.device)
                self._workspace(B, T, n)
                torch.cuda.synchronize(self.device)
                s = torch.cuda.Stream(self.device)
                s.wait_stream(torch.cuda.current_stream(self.device))
                with torch.cuda.stream(s):
                    self._call(self._g_in, self._g_st, self._g_gl, self._g_out, self._g_cost)  # warm-up
                torch.cuda.current_stream(self.device).wait_stream(s)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._call(self._g_in, self._g_st, self._g_gl, self._g_out, self._g_cost)
                self._graph = g
            self._g_in.copy_(init)
            self._g_st.copy_(st)
            self._g_gl.copy_(gl)
            self._graph.replay()
            out, costs = self._g_out, self._g_cost
        return out[int(torch.argmin(costs))], costs, out

    def launches_per_run(self) -> int:
        """Kernel launches of one ``run``: pin, per outer (linearise [+ 2 FD kernels], inner), final (2)."""
        per = 2 + (2 if self.opt.fd_eps > 0 else 0)
        return 1 + self.cfg.n_outer_iters * per + 2


def sco_trajopt(init_trajs, start, goal, model: RobotModel, spheres: RobotSpheres, world, link_pairs,
                cfg: ScoConfig = ScoConfig(), *, fd_eps: float = 0.0, self_all_pairs: bool = True, device="cuda"):
    """Functional form of ``sco_trajopt(..., use_cuda=True)``."""
    opt = ScoOptimizer(model, spheres, world, link_pairs, cfg, fd_eps=fd_eps, self_all_pairs=self_all_pairs,
                       device=device)
    return opt.run(torch.as_tensor(init_trajs, device=opt.device), torch.as_tensor(start, device=opt.device),
                   torch.as_tensor(goal, device=opt.device))


def make_init_trajs(start, goal, n_batch: int, n_timesteps: int, seed: int = 0, noise_scale: float = 0.05):
    """Linear interpolation plus Gaussian noise (``make_init_trajs``, ``_sco_optimization.py:554-564``;
    numpy's generator stands in for ``jax.random``)."""
    start = np.asarray(start, np.float64)
    goal = np.asarray(goal, np.float64)
    t = np.linspace(0.0, 1.0, n_timesteps)[:, None]
    base = start[None] * (1.0 - t) + goal[None] * t
    trajs = np.broadcast_to(base[None], (n_batch, n_timesteps, start.shape[0]))
    noise = np.random.default_rng(seed).normal(size=trajs.shape) * noise_scale
    return (trajs + noise).astype(np.float32)
