"""GPU CHOMP loop (``pyroffi_b200.chomp``) against the FP64 oracle loop, and
CUDA-graph replay against the eager run."""

import numpy as np
import pytest
import torch

from oracle import chomp as ochomp
from pyroffi_b200 import workloads as W
from pyroffi_b200.chomp import ChompConfig, ChompOptimizer, cg_solve
from pyroffi_b200.trajopt import TrajectoryCost

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def small():
    w = W.trajectories(Bt=3, T=12)
    return w


def test_cg_matches_oracle():
    rng = np.random.default_rng(0)
    b = rng.normal(size=(5, 20))
    got = cg_solve(torch.as_tensor(b, dtype=torch.float64, device=DEV), 1e-3, 24, 1e-4).cpu().numpy()
    for i in range(5):
        np.testing.assert_allclose(got[i], ochomp.cg_solve(b[i].copy(), 1e-3, 24, 1e-4), rtol=1e-8, atol=1e-10)


@pytest.mark.parametrize("n_iters", [1, 3])
def test_chomp_steps_match_oracle(n_iters):
    w = small()
    cfg = ChompConfig(n_iters=n_iters)
    tc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=cfg.collision_margin, device=DEV)
    start, goal = w.traj[0, 0], w.traj[0, -1]
    init = w.traj.copy()
    init[:, 0], init[:, -1] = start, goal
    best, costs, final = ChompOptimizer(tc, cfg).run(torch.as_tensor(init, device=DEV),
                                                      torch.as_tensor(start, device=DEV),
                                                      torch.as_tensor(goal, device=DEV))
    final = final.cpu().numpy()
    m = w.model.as_dict()
    centers, radii = w.spheres.centers, w.spheres.radii
    world = w.world.arrays()
    for b in range(init.shape[0]):
        ox, _ = ochomp.chomp_single(init[b], start, goal, m, centers, radii, w.link_pairs, world, w.model.lower,
                                    w.model.upper, cfg)
        np.testing.assert_allclose(final[b], ox, atol=2e-4)


def test_chomp_graph_replay_equals_eager():
    w = W.trajectories(Bt=8, T=24)
    cfg = ChompConfig(n_iters=10)
    tc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=cfg.collision_margin, device=DEV)
    x = torch.as_tensor(w.traj, device=DEV)
    s, g = x[0, 0].clone(), x[0, -1].clone()
    opt = ChompOptimizer(tc, cfg)
    b1, c1, f1 = opt.run(x, s, g)
    b2, c2, f2 = opt.run(x, s, g, graph=True)
    b3, c3, f3 = opt.run(x, s, g, graph=True)
    torch.testing.assert_close(f2, f1, rtol=0, atol=0)
    torch.testing.assert_close(f3, f1, rtol=0, atol=0)
    assert torch.all(c1 <= tc_cost_initial(tc, x, cfg) + 1e-3)


def tc_cost_initial(tc, x, cfg):
    xx = x.clone()
    xx[:, 0], xx[:, -1] = x[0, 0], x[0, -1]
    tc.opt.w_coll = cfg.w_collision_max
    return tc.cost(xx)
