"""LM penalty terms beyond world spheres, against the FP64 oracle: capsule,
box and halfspace obstacles and explicit self sphere pairs, for the
seed-group body (7-DOF chain) and the warp-per-seed body (15-DOF bimanual
tree, two hand targets), a few iterations seed by seed."""

import numpy as np
import pytest
import torch

from oracle import kinematics as okin
from oracle import lm as olm
from pyroffi_b200 import robot as R
from pyroffi_b200 import workloads as W
from pyroffi_b200.ik import BatchIkSolver

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def tt(x):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float32, device=DEV)


def mixed_world(rng):
    w = W.empty_world()
    w.spheres = W.random_sphere_world(rng, 30)
    w.capsules = np.concatenate([rng.uniform(-1, 1, (4, 6)), rng.uniform(0.02, 0.1, (4, 1))], 1).astype(np.float32)
    w.boxes = W.random_boxes(rng, 5, oriented=True)
    n = rng.normal(size=(2, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    w.halfspaces = np.concatenate([n, rng.uniform(-1, 1, (2, 3))], 1).astype(np.float32)
    return w


@pytest.mark.parametrize("robot,tps", [("chain7", 2), ("chain7", 4), ("chain7", 16), ("bimanual", 16), ("bimanual", 32)])
@pytest.mark.parametrize("max_iter", [0, 1, 2])
def test_lm_mixed_world_and_self_pairs(robot, tps, max_iter):
    rng = np.random.default_rng(21)
    if robot == "chain7":
        model = R.serial_chain(7, rng)
        links = (model.n_links - 1,)
    else:
        model = R.bimanual_tree(rng)
        links = (10, 16)
    spheres = R.random_spheres(model, rng, per_link=4)
    rs, jidx, link_of = spheres.flat_for_ik(model)
    pairs = W.self_sphere_pairs(link_of, model, 40, rng)
    world = mixed_world(rng)
    P, Sd = 2, 20
    tcfg = model.random_cfgs(rng, P).astype(np.float64)
    Tj = okin.fk_joints(tcfg, model.twists, model.parent_tf, model.parent_idx, model.act_idx, model.mimic_mul,
                        model.mimic_off, model.mimic_act_idx, model.topo_inv)
    tj = [model.link_joint(l) for l in links]
    target = Tj[:, tj]                                           # [P, n_ee, 7]
    seeds = rng.uniform(model.lower, model.upper, size=(P, Sd, model.n_act)).astype(np.float32)
    opts = dict(max_iter=max_iter, lambda_init=1e-2, lambda_down=0.1, lambda_up=10.0, collision_weight=1e3,
                collision_margin=0.05)
    s = BatchIkSolver(model, links, spheres=spheres, world=world, self_pairs=pairs, threads_per_seed=tps,
                      device=DEV, **opts)
    cfgs, errs = s.run_lm(tt(target), tt(seeds))
    cfgs, errs = cfgs.cpu().numpy(), errs.cpu().numpy()
    ok = 0
    for p in range(P):
        oc, oe = olm.ls_ik(seeds[p], target[p][None], model.as_dict(), tj, [model.ancestor_mask(l) for l in links],
                           lower=model.lower, upper=model.upper, max_iter=max_iter, lambda_init=1e-2,
                           lambda_down=0.1, lambda_up=10.0, enable_collision=True, collision_weight=1e3,
                           collision_margin=0.05, spheres_local=rs, sphere_joint=jidx, ws=world.spheres,
                           wc=world.capsules, wb=world.boxes, wh=world.halfspaces, self_i=pairs[:, 0],
                           self_j=pairs[:, 1])
        close = (np.abs(cfgs[p] - oc).max(axis=1) < 2e-4) & (np.abs(errs[p] - oe) <= 1e-3 * np.abs(oe) + 1e-4)
        ok += int(close.sum())
        if max_iter == 0:
            np.testing.assert_allclose(errs[p], oe, rtol=3e-5, atol=1e-5)
    assert ok >= 0.9 * P * Sd, ok
