"""GPU SQP-IK (``pk_sqp_ik_cuda``, ``pyroffi_b200.sqp``) against the FP64
oracle (``oracle/sqp.py``): the scores at the seeds, the iterations seed by
seed (agreement rate; a line-search or active-set choice may flip in FP32),
joint limits as hard bounds, fixed joints, a two-EE robot, and the solve's
success against the oracle run on the same seeds."""

import numpy as np
import pytest
import torch

from oracle import lm as olm
from oracle import sqp as osqp
from pyroffi_b200 import workloads as W
from pyroffi_b200.sqp import SqpSolver

from ik_cases import agree, bimanual, t

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
KW = dict(n_inner_iters=2, pos_weight=50.0, ori_weight=10.0, lambda_init=5e-3)   # tests/bench_ik.py:220-233
OKW = dict(n_inner=2, pos_weight=50.0, ori_weight=10.0, lambda_init=5e-3, eps_pos=1e-8, eps_ori=1e-8)


def chain(P=3, S=32, seed=1002, coll=False):
    w = W.ik(P=P, Sd=S, seed=seed)
    sol = SqpSolver(w.model, w.target_link, spheres=w.spheres, world=w.world, enable_collision=coll, device=DEV)
    tj = [w.model.link_joint(w.target_link)]
    anc = [w.model.ancestor_mask(w.target_link)]
    oc = None
    if coll:
        oc = dict(world=w.world.arrays(), spheres_local=w.spheres_local, sphere_joint=w.sphere_joint, margin=0.02,
                  weight=1e4)
    return w, sol, tj, anc, w.target_T[:, None, :], oc


@pytest.mark.parametrize("coll", [False, True])
def test_scores_at_the_seeds(coll):
    w, sol, tj, anc, tgt, oc = chain(coll=coll)
    _, err = sol.run(t(w.seeds), t(w.target_T), max_iter=0, **KW)
    for p in range(w.seeds.shape[0]):
        _, oe = osqp.sqp(w.seeds[p], tgt[p:p + 1], w.model.as_dict(), tj, anc, w.model.lower, w.model.upper,
                         np.zeros(w.model.n_act, bool), max_iter=0, coll=oc, **OKW)
        np.testing.assert_allclose(err.cpu().numpy()[p], oe, rtol=2e-5, atol=1e-6)


@pytest.mark.parametrize("coll,iters", [(False, 3), (False, 20), (True, 8)])
def test_iterations_match_oracle(coll, iters):
    w, sol, tj, anc, tgt, oc = chain(coll=coll)
    cfg, err = sol.run(t(w.seeds), t(w.target_T), max_iter=iters, **KW)
    cfg, err = cfg.cpu().numpy(), err.cpu().numpy()
    rates = []
    for p in range(w.seeds.shape[0]):
        _, oe = osqp.sqp(w.seeds[p], tgt[p:p + 1], w.model.as_dict(), tj, anc, w.model.lower, w.model.upper,
                         np.zeros(w.model.n_act, bool), max_iter=iters, coll=oc, **OKW)
        rates.append(agree(err[p], oe, rtol=1e-2, atol=1e-6))
        assert np.all(cfg[p] >= w.model.lower - 1e-6) and np.all(cfg[p] <= w.model.upper + 1e-6)
    assert np.mean(rates) >= 0.85, rates


def test_fixed_joints_and_limits():
    w, sol, *_ = chain(S=16)
    mask = np.zeros(w.model.n_act, np.int32)
    mask[[0, 5]] = 1
    sol.set_fixed_mask(mask)
    cfg, _ = sol.run(t(w.seeds), t(w.target_T), max_iter=15, **KW)
    cfg = cfg.cpu().numpy()
    np.testing.assert_array_equal(cfg[..., [0, 5]], w.seeds[..., [0, 5]])
    assert np.all(cfg >= w.model.lower - 1e-6) and np.all(cfg <= w.model.upper + 1e-6)


@pytest.mark.parametrize("links", [None, (10, 16, 7)])
def test_two_end_effectors_match_oracle(links):
    """Two hands (the 2-EE kernel), and the hands plus an elbow (the 4-EE kernel)."""
    m, sol, tj, anc, tgt, seeds = bimanual(target_links=links, solver=SqpSolver)
    _, e0 = sol.run(t(seeds), t(tgt), max_iter=0, **KW)
    _, e1 = sol.run(t(seeds), t(tgt), max_iter=6, **KW)
    fixed = np.zeros(m.n_act, bool)
    rates = []
    for p in range(seeds.shape[0]):
        _, oe0 = osqp.sqp(seeds[p], tgt[p:p + 1], m.as_dict(), tj, anc, m.lower, m.upper, fixed, max_iter=0, **OKW)
        np.testing.assert_allclose(e0.cpu().numpy()[p], oe0, rtol=2e-5, atol=1e-6)
        _, oe1 = osqp.sqp(seeds[p], tgt[p:p + 1], m.as_dict(), tj, anc, m.lower, m.upper, fixed, max_iter=6, **OKW)
        rates.append(agree(e1.cpu().numpy()[p], oe1, rtol=1e-2, atol=1e-6))
    assert np.mean(rates) >= 0.85, rates


def test_solve_matches_oracle_on_the_same_seeds():
    P = 16
    w, sol, tj, anc, tgt, _ = chain(P=P, S=8)
    g = torch.Generator(device=DEV).manual_seed(0)
    prev = t(w.model.random_cfgs(np.random.default_rng(9), P))
    best, _, (seeds, cfg, err) = sol.solve(t(w.target_T), prev, num_seeds=32, max_iter=60, generator=g,
                                           return_all=True, **KW)
    seeds, cfg, err = seeds.cpu().numpy(), cfg.cpu().numpy(), err.cpu().numpy()
    np.testing.assert_array_equal(best.cpu().numpy(), cfg[np.arange(P), np.argmin(err, axis=1)])
    md = w.model.as_dict()
    ok_gpu, ok_or = [], []
    for p in range(P):
        ocfg, oerr = osqp.sqp(seeds[p], tgt[p:p + 1], md, tj, anc, w.model.lower, w.model.upper,
                              np.zeros(w.model.n_act, bool), max_iter=60, **OKW)
        for c, acc in ((best.cpu().numpy()[p], ok_gpu), (ocfg[np.argmin(oerr)], ok_or)):
            pe, re = olm.pose_errors(c[None].astype(np.float64), w.target_T[p:p + 1], md, tj[0])
            acc.append(bool(pe[0] < 1e-3 and re[0] < 1e-2))
    assert np.mean(ok_gpu) >= 0.8
    assert abs(np.mean(ok_gpu) - np.mean(ok_or)) <= 0.15, (np.mean(ok_gpu), np.mean(ok_or))


def test_partial_seed_blocks_and_empty_batch():
    """33 seeds: a full 32-seed block and a block of one; no problems at all."""
    w, sol, tj, anc, tgt, oc = chain(P=2, S=33, coll=True)
    cfg, err = sol.run(t(w.seeds), t(w.target_T), max_iter=5, **KW)
    cfg, err = cfg.cpu().numpy(), err.cpu().numpy()
    for p in range(2):
        _, oe = osqp.sqp(w.seeds[p], tgt[p:p + 1], w.model.as_dict(), tj, anc, w.model.lower, w.model.upper,
                         np.zeros(w.model.n_act, bool), max_iter=5, coll=oc, **OKW)
        assert agree(err[p], oe) >= 0.85
        assert np.all(cfg[p] >= w.model.lower - 1e-6) and np.all(cfg[p] <= w.model.upper + 1e-6)
    c0, e0 = sol.run(t(w.seeds[:0]), t(w.target_T[:0]), max_iter=5, **KW)
    assert c0.shape == (0, 33, w.model.n_act) and e0.shape == (0, 33)
