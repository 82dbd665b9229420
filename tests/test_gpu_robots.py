"""Kernels on a robot the reference ships: the spherized Panda (parsed from
its URDF + SRDF into ``tests/golden/robots/panda.npz`` by
``tests/golden/make_robot_fixtures.py``).  FK and link poses, self distances
of the SRDF's active link pairs, the fused FK -> sphere -> world distances,
the trajectory cost, and LM / HJCD / SQP IK to the hand, each against the
FP64 oracle or the FP64 success test."""

import numpy as np
import pytest
import torch

from oracle import collision as ocoll
from oracle import kinematics as okin
from oracle import lm as olm
from oracle import traj as otraj
from pyroffi_b200 import workloads as W
from pyroffi_b200.collision import fk_sphere_collision
from pyroffi_b200.cuda_kernels import collision_self_sphere, fk_cuda
from pyroffi_b200.device import DeviceRobot, DeviceSpheres, DeviceWorld
from pyroffi_b200.hjcd import HjcdSolver
from pyroffi_b200.ik import BatchIkSolver
from pyroffi_b200.sqp import SqpSolver
from pyroffi_b200.trajopt import TrajectoryCost

from error_report import assert_distances
from robot_fixtures import load_robot

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def t(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=DEV)


@pytest.fixture(scope="module")
def panda():
    return load_robot("panda")


def test_fk_and_link_poses(panda):
    m, *_ = panda
    cfg = m.random_cfgs(np.random.default_rng(0), 256)
    Tj = fk_cuda(t(cfg), t(m.twists), t(m.parent_tf), t(m.parent_idx, torch.int32), t(m.act_idx, torch.int32),
                 t(m.mimic_mul), t(m.mimic_off), t(m.mimic_act_idx, torch.int32), t(m.topo_inv, torch.int32),
                 t(m.fk_level_starts, torch.int32), t(m.fk_level_joints, torch.int32)).cpu().numpy()
    md = m.as_dict()
    ref = okin.fk_joints(cfg.astype(np.float64), md["twists"], md["parent_tf"], md["parent_idx"], md["act_idx"],
                         md["mimic_mul"], md["mimic_off"], md["mimic_act_idx"], md["topo_inv"])
    np.testing.assert_allclose(Tj[..., 4:], ref[..., 4:], atol=1e-5)
    dots = np.abs(np.sum(Tj[..., :4] * ref[..., :4], axis=-1))
    assert np.all(dots > 1 - 1e-6)


def test_self_distances_of_the_srdf_pairs(panda):
    m, sp, pairs, _ = panda
    cfg = m.random_cfgs(np.random.default_rng(1), 128).astype(np.float64)
    links = okin.forward_kinematics(cfg, m.as_dict())                       # [B, N, 7]
    cen = ocoll.transform_points(links[:, :, None, :], sp.centers.astype(np.float64)[None])   # [B, N, S, 3]
    c_bsn3 = np.ascontiguousarray(cen.transpose(0, 2, 1, 3))
    r_bsn = np.ascontiguousarray(np.broadcast_to(sp.radii.T[None], c_bsn3.shape[:-1]))
    got = collision_self_sphere(t(c_bsn3), t(r_bsn), t(pairs[:, 0], torch.int32),
                                t(pairs[:, 1], torch.int32)).cpu().numpy()
    want = ocoll.self_sphere_full(c_bsn3, r_bsn, pairs[:, 0], pairs[:, 1])
    assert_distances(got, want, quantity="signed distance (collision_self_sphere)", case="panda SRDF pairs")


def test_fused_world_distances(panda):
    m, sp, _, _ = panda
    rng = np.random.default_rng(2)
    world = W.empty_world()
    world.spheres = W.random_sphere_world(rng, 64)
    world.boxes = W.random_boxes(rng, 8, oriented=True)
    cfg = m.random_cfgs(rng, 256)
    r = fk_sphere_collision(DeviceRobot.upload(m, DEV), DeviceSpheres.upload(sp, DEV), DeviceWorld.upload(world, DEV),
                            t(cfg), per_link=True)
    links = okin.forward_kinematics(cfg.astype(np.float64), m.as_dict())
    cen = ocoll.transform_points(links[:, :, None, :], sp.centers.astype(np.float64)[None])
    d = ocoll.point_vs_world(cen, np.broadcast_to(sp.radii, cen.shape[:-1]), *world.arrays())   # [B, N, S, M]
    d = np.where(sp.radii[None, :, :, None] < 0, np.inf, d).min(axis=2)                        # [B, N, M]
    got = r.dist_bnm.cpu().numpy()
    fin = np.isfinite(d)
    assert_distances(got[fin], d[fin], quantity="signed distance (fused, per link)", case="panda")
    assert_distances(r.min_dist.cpu().numpy(), np.where(fin, d, np.inf).reshape(256, -1).min(axis=1),
                     quantity="signed distance (fused, minimum)", case="panda")


def test_trajectory_cost_and_gradient(panda):
    m, sp, pairs, _ = panda
    rng = np.random.default_rng(3)
    world = W.empty_world()
    world.spheres = W.random_sphere_world(rng, 32)
    start, goal = m.random_cfgs(rng, 1)[0], m.random_cfgs(rng, 1)[0]
    s = np.linspace(0, 1, 16)[:, None]
    traj = (start * (1 - s) + goal * s)[None].astype(np.float32)
    tc = TrajectoryCost(m, sp, world, pairs, device=DEV)
    c, g = tc.cost_and_grad(t(traj))
    o = tc.opt
    want = otraj.total_cost(traj[0], m.as_dict(), sp.centers, sp.radii, pairs, world.arrays(), margin=o.margin,
                            w_smooth=o.w_smooth, w_acc=o.w_acc, w_jerk=o.w_jerk, w_limits=o.w_limits, w_coll=o.w_coll,
                            lower=m.lower, upper=m.upper)
    np.testing.assert_allclose(float(c[0]), want, rtol=1e-4, atol=1e-6)
    assert torch.isfinite(g).all()


@pytest.mark.parametrize("solver", ["lm", "hjcd", "sqp"])
def test_ik_to_the_hand(panda, solver):
    m, sp, _, ee = panda
    rng = np.random.default_rng(4)
    P = 32
    goal_cfg = m.random_cfgs(rng, P)
    links = okin.forward_kinematics(goal_cfg.astype(np.float64), m.as_dict())
    tgt = links[:, ee].astype(np.float32)                                     # [P, 7]
    prev = m.random_cfgs(rng, P)
    g = torch.Generator(device=DEV).manual_seed(0)
    if solver == "lm":
        s = BatchIkSolver(m, ee, max_iter=60, device=DEV)
        best = s.solve(t(tgt), s.make_seeds(t(prev), 64, g)).winner_cfg
    elif solver == "hjcd":
        best = HjcdSolver(m, ee, device=DEV).solve(t(tgt), t(prev), num_seeds=32, lambda_init=1e-3,
                                                    limit_prior_weight=1e-4, kick_scale=0.02, generator=g)
    else:
        best = SqpSolver(m, ee, device=DEV).solve(t(tgt), t(prev), num_seeds=32, generator=g)
    pe, re = olm.pose_errors(best.cpu().numpy().astype(np.float64), tgt, m.as_dict(), m.link_joint(ee))
    ok = (pe < 1e-3) & (re < 1e-2)
    assert ok.mean() >= 0.8, (solver, ok.mean(), np.median(pe), np.median(re))
