"""GPU CHOMP loop (``pyroffi_b200.chomp``) against the FP64 oracle loop, and
CUDA-graph replay against the eager run."""

import numpy as np
import pytest
import torch

from oracle import chomp as ochomp
from pyroffi_b200 import workloads as W
from pyroffi_b200.chomp import ChompConfig, ChompOptimizer, covariant_direction
from pyroffi_b200.trajopt import TrajectoryCost

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def small():
    w = W.trajectories(Bt=3, T=12)
    return w


@pytest.mark.parametrize("T,n,clip,covariant", [(64, 7, 10.0, True), (12, 3, 0.0, True), (130, 9, 0.5, True),
                                                (20, 4, 10.0, False)])
def test_direction_kernel_matches_oracle(T, n, clip, covariant):
    # clipping, pinned ends and the FP64 truncated CG of every joint timeline
    rng = np.random.default_rng(T + n)
    g = (rng.normal(size=(5, T, n)) * rng.uniform(0.1, 10.0, size=(5, 1, 1))).astype(np.float32)
    g[1, :, 0] *= 1e-9                                            # a timeline that stops after one step
    cfg = ChompConfig(grad_clip_norm=clip, use_covariant_update=covariant)
    got = covariant_direction(torch.as_tensor(g, device=DEV), cfg).cpu().numpy()
    for b in range(5):
        gb = g[b].astype(np.float64)
        gn = np.sqrt(np.sum(g[b].astype(np.float64) ** 2))
        if clip > 0 and gn > clip:
            gb = gb * (clip / (gn + 1e-12))
        want = np.zeros_like(gb)
        for j in range(n):
            if covariant:
                want[1:-1, j] = -ochomp.cg_solve(gb[1:-1, j].copy(), cfg.smoothness_reg, cfg.n_cg_iters, cfg.cg_tol)
            else:
                want[1:-1, j] = -gb[1:-1, j]
        np.testing.assert_allclose(got[b], want, rtol=1e-5, atol=1e-6 * (np.abs(want).max() + 1e-30))
        assert np.all(got[b, 0] == 0) and np.all(got[b, -1] == 0)


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


def test_line_search_kernels_match_the_tensor_formulation():
    """pk_chomp_line_trials / pk_chomp_line_select against the same step in
    torch ops: trials, first minimum, improvement test, stall count, early stop."""
    from pyroffi_b200 import _lib
    from pyroffi_b200._tensors import ptr, stream_ptr
    rng = np.random.default_rng(4)
    K, B, T, n = 5, 37, 9, 7
    tr = torch.as_tensor(rng.normal(size=(B, T, n)), dtype=torch.float32, device=DEV)
    d = torch.as_tensor(rng.normal(size=(B, T, n)) * 2.0, dtype=torch.float32, device=DEV)
    alphas = torch.tensor([1.0, 0.5, 0.25, 0.1, 0.05], dtype=torch.float32, device=DEV) * 0.7
    start = torch.as_tensor(rng.normal(size=n), dtype=torch.float32, device=DEV)
    goal = torch.as_tensor(rng.normal(size=n), dtype=torch.float32, device=DEV)
    md = 0.3
    trials = torch.empty((K, B, T, n), dtype=torch.float32, device=DEV)
    st = stream_ptr(torch.device(DEV))
    _lib.call("pk_chomp_line_trials", st, ptr(tr), ptr(d), ptr(alphas), K, md, ptr(start), ptr(goal), ptr(trials),
              B, T, n, None)
    ref = tr[None] + torch.clamp(alphas[:, None, None, None] * d[None], -md, md)
    ref[:, :, 0] = start
    ref[:, :, -1] = goal
    assert torch.equal(trials, ref)

    c = torch.as_tensor(rng.uniform(1.0, 2.0, size=B), dtype=torch.float32, device=DEV)
    tc = torch.as_tensor(rng.uniform(0.9, 2.1, size=(K, B)), dtype=torch.float32, device=DEV)
    tc[:, :5] = c[:5]                                        # ties with the current cost: no step
    tc[2, 5:9] = tc[1, 5:9]                                  # ties between trials: the first wins
    active = torch.as_tensor(rng.uniform(size=B) < 0.8, device=DEV)
    stall = torch.as_tensor(rng.integers(0, 4, size=B), dtype=torch.int32, device=DEV)
    mci, pat = 1e-5, 3
    # torch formulation of the step
    tcc = torch.cat([tc, c[None]], dim=0)
    tall = torch.cat([trials, tr[None]], dim=0)
    best_cost, best_idx = torch.min(tcc, dim=0)
    best = tall[best_idx, torch.arange(B, device=DEV)]
    improved = best_cost < (c - mci)
    want_tr = torch.where((active & improved)[:, None, None], best, tr)
    want_stall = torch.where(active, torch.where(improved, torch.zeros_like(stall), stall + 1), stall)
    want_active = active & (want_stall < pat)
    _lib.call("pk_chomp_line_select", st, ptr(tc), ptr(c), ptr(trials), ptr(tr), ptr(active), ptr(stall), K, mci,
              pat, B, T, n)
    assert torch.equal(tr, want_tr)
    assert torch.equal(stall, want_stall)
    assert torch.equal(active, want_active)


def test_skipping_finished_trajectories_leaves_results_unchanged():
    """Early-stopped trajectories no longer change, so the cost, gradient,
    direction and trial launches skip them (the kernels' active masks); on
    the config-3 trajectories, where most stop within 100 iterations, the
    final trajectories and costs are the same bits with and without the skip."""
    wt = W.trajectories(Bt=64, T=64)
    cfg = ChompConfig()
    x = torch.as_tensor(wt.traj, device=DEV)
    s0, g0 = x[0, 0].clone(), x[0, -1].clone()
    out = []
    for skip in (True, False):
        tc = TrajectoryCost(wt.model, wt.spheres, wt.world, wt.link_pairs, margin=cfg.collision_margin, device=DEV)
        _, costs, final = ChompOptimizer(tc, cfg, skip_finished=skip).run(x, s0, g0)
        out.append((costs.clone(), final.clone()))
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])


def test_masked_kernels_write_only_active_rows():
    from pyroffi_b200 import _lib
    from pyroffi_b200._tensors import ptr, stream_ptr
    rng = np.random.default_rng(3)
    K, B, T, n = 2, 9, 8, 5
    tr = torch.as_tensor(rng.normal(size=(B, T, n)), dtype=torch.float32, device=DEV)
    d = torch.as_tensor(rng.normal(size=(B, T, n)), dtype=torch.float32, device=DEV)
    alphas = torch.tensor([1.0, 0.5], dtype=torch.float32, device=DEV)
    start, goal = tr[0, 0].clone(), tr[0, -1].clone()
    active = torch.as_tensor(np.arange(B) % 3 != 1, device=DEV)
    trials = torch.full((K, B, T, n), 7.0, dtype=torch.float32, device=DEV)
    _lib.call("pk_chomp_line_trials", stream_ptr(torch.device(DEV)), ptr(tr), ptr(d), ptr(alphas), K, 0.3,
              ptr(start), ptr(goal), ptr(trials), B, T, n, ptr(active))
    ref = torch.full_like(trials, 7.0)
    _lib.call("pk_chomp_line_trials", stream_ptr(torch.device(DEV)), ptr(tr), ptr(d), ptr(alphas), K, 0.3,
              ptr(start), ptr(goal), ptr(ref), B, T, n, None)
    a = active.cpu().numpy()
    assert torch.equal(trials[:, a], ref[:, a])
    assert torch.all(trials[:, ~a] == 7.0)
    g = torch.as_tensor(rng.normal(size=(B, 12, n)), dtype=torch.float32, device=DEV)
    full = covariant_direction(g, ChompConfig())
    part = covariant_direction(g, ChompConfig(), active)
    assert torch.equal(part[a], full[a])
