"""GPU HJCD-IK (``pk_hjcd_ik_coarse_cuda``, ``pk_hjcd_ik_lm_cuda``,
``pyroffi_b200.hjcd``) against the FP64 oracle (``oracle/hjcd.py``): the
scores at the seeds exactly, the coarse and refinement iterations seed by
seed (agreement rate: a near-tie in a discrete choice -- the greedy joint, a
line-search step -- may go the other way in FP32), the stop flag, fixed
joints, a two-EE robot, and the whole solve's success rate."""

import numpy as np
import pytest
import torch

from oracle import hjcd as ohjcd
from oracle import lm as olm
from pyroffi_b200 import workloads as W
from pyroffi_b200.hjcd import HjcdSolver

from ik_cases import agree, bimanual, t

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
REF_KW = dict(lambda_init=1e-3, limit_prior_weight=1e-4, kick_scale=0.02)   # tests/bench_ik.py:193-201


def chain(P=3, S=32, seed=1002, coll=False):
    w = W.ik(P=P, Sd=S, seed=seed)
    sol = HjcdSolver(w.model, w.target_link, spheres=w.spheres, world=w.world, enable_collision=coll, device=DEV)
    tj = [w.model.link_joint(w.target_link)]
    anc = [w.model.ancestor_mask(w.target_link)]
    tgt = w.target_T[:, None, :]
    oc = None
    if coll:
        oc = dict(world=w.world.arrays(), spheres_local=w.spheres_local, sphere_joint=w.sphere_joint, margin=0.02,
                  weight=1e4)
    return w, sol, tj, anc, tgt, oc


@pytest.mark.parametrize("coll", [False, True])
def test_scores_at_the_seeds_match(coll):
    w, sol, tj, anc, tgt, oc = chain(coll=coll)
    _, err = sol.coarse(t(w.seeds), t(w.target_T), k_max=0)
    err = err.cpu().numpy()
    for p in range(w.seeds.shape[0]):
        _, oe = ohjcd.coarse(w.seeds[p], tgt[p:p + 1], w.model.as_dict(), tj, anc, w.model.lower, w.model.upper,
                             np.zeros(w.model.n_act, bool), 0, coll=oc)
        np.testing.assert_allclose(err[p], oe, rtol=2e-5, atol=1e-7)


@pytest.mark.parametrize("coll", [False, True])
def test_coarse_descent_matches_oracle(coll):
    w, sol, tj, anc, tgt, oc = chain(coll=coll)
    cfg, err = sol.coarse(t(w.seeds), t(w.target_T), k_max=20)
    cfg, err = cfg.cpu().numpy(), err.cpu().numpy()
    rates = []
    for p in range(w.seeds.shape[0]):
        ocfg, oe = ohjcd.coarse(w.seeds[p], tgt[p:p + 1], w.model.as_dict(), tj, anc, w.model.lower, w.model.upper,
                                np.zeros(w.model.n_act, bool), 20, coll=oc)
        rates.append(agree(err[p], oe))
        assert np.all(cfg[p] >= w.model.lower - 1e-6) and np.all(cfg[p] <= w.model.upper + 1e-6)
    assert np.mean(rates) >= 0.9, rates


@pytest.mark.parametrize("coll,iters", [(False, 5), (False, 20), (True, 10)])
def test_refinement_matches_oracle(coll, iters):
    w, sol, tj, anc, tgt, oc = chain(coll=coll, S=30)
    ccfg, _ = sol.coarse(t(w.seeds), t(w.target_T), k_max=20)
    noise = np.random.default_rng(5).normal(size=(w.seeds.shape[0], 30, iters, w.model.n_act)).astype(np.float32)
    cfg, err, stop = sol.refine(ccfg, t(noise), t(w.target_T), max_iter=iters, **REF_KW)
    cfg, err = cfg.cpu().numpy(), err.cpu().numpy()
    seeds = ccfg.cpu().numpy()
    rates = []
    for p in range(w.seeds.shape[0]):
        ocfg, oe, ostop = ohjcd.lm_refine(seeds[p], noise[p], tgt[p:p + 1], w.model.as_dict(), tj, anc,
                                          w.model.lower, w.model.upper, np.zeros(w.model.n_act, bool),
                                          max_iter=iters, stall_patience=6, eps_pos=1e-8, eps_ori=1e-8, coll=oc,
                                          **REF_KW)
        rates.append(agree(err[p], oe, rtol=1e-2, atol=1e-8))
        assert int(stop[p]) == int(ostop) == 0
    assert np.mean(rates) >= 0.85, rates


def test_stop_flag_ends_every_seed_of_the_problem():
    w, sol, tj, anc, tgt, _ = chain(S=20)
    noise = t(np.zeros((w.seeds.shape[0], 20, 5, w.model.n_act)))
    cfg, err, stop = sol.refine(t(w.seeds), noise, t(w.target_T), max_iter=5, eps_pos=10.0, eps_ori=10.0, **REF_KW)
    assert torch.all(stop == 1)
    np.testing.assert_array_equal(cfg.cpu().numpy(), w.seeds)        # stopped before the first step
    _, e0 = sol.coarse(t(w.seeds), t(w.target_T), k_max=0)   # the same score from the other kernel
    np.testing.assert_allclose(err.cpu().numpy(), e0.cpu().numpy(), rtol=1e-6)


def test_fixed_joints_do_not_move():
    w, sol, *_ = chain(S=16)
    mask = np.zeros(w.model.n_act, np.int32)
    mask[[1, 4]] = 1
    sol.set_fixed_mask(mask)
    cfg, _ = sol.coarse(t(w.seeds), t(w.target_T), k_max=10)
    np.testing.assert_array_equal(cfg.cpu().numpy()[..., [1, 4]], w.seeds[..., [1, 4]])
    noise = t(np.random.default_rng(2).normal(size=(w.seeds.shape[0], 16, 12, w.model.n_act)))
    c2, _, _ = sol.refine(t(w.seeds), noise, t(w.target_T), max_iter=12, stall_patience=2, lambda_init=1e-3,
                          limit_prior_weight=1e-4, kick_scale=0.5)
    np.testing.assert_array_equal(c2.cpu().numpy()[..., [1, 4]], w.seeds[..., [1, 4]])


@pytest.mark.parametrize("links", [None, (10, 16, 7)])
def test_two_end_effectors_match_oracle(links):
    """Two hands (the 2-EE kernels), and the hands plus an elbow (the 4-EE kernels)."""
    m, sol, tj, anc, tgt, seeds = bimanual(target_links=links)
    _, e0 = sol.coarse(t(seeds), t(tgt), k_max=0)
    cfg, err = sol.coarse(t(seeds), t(tgt), k_max=15)
    noise = np.random.default_rng(3).normal(size=(seeds.shape[0], seeds.shape[1], 8, m.n_act)).astype(np.float32)
    rcfg, rerr, _ = sol.refine(cfg, t(noise), t(tgt), max_iter=8, **REF_KW)
    e0, err, rerr, cfg = e0.cpu().numpy(), err.cpu().numpy(), rerr.cpu().numpy(), cfg.cpu().numpy()
    md = m.as_dict()
    fixed = np.zeros(m.n_act, bool)
    r1, r2 = [], []
    for p in range(seeds.shape[0]):
        _, oe0 = ohjcd.coarse(seeds[p], tgt[p:p + 1], md, tj, anc, m.lower, m.upper, fixed, 0)
        np.testing.assert_allclose(e0[p], oe0, rtol=2e-5, atol=1e-7)
        _, oe = ohjcd.coarse(seeds[p], tgt[p:p + 1], md, tj, anc, m.lower, m.upper, fixed, 15)
        r1.append(agree(err[p], oe))
        _, ore, _ = ohjcd.lm_refine(cfg[p], noise[p], tgt[p:p + 1], md, tj, anc, m.lower, m.upper, fixed, max_iter=8,
                                    stall_patience=6, eps_pos=1e-8, eps_ori=1e-8, **REF_KW)
        r2.append(agree(rerr[p], ore, rtol=1e-2, atol=1e-8))
    assert np.mean(r1) >= 0.9 and np.mean(r2) >= 0.85, (r1, r2)


def test_solve_matches_oracle_refinement_of_the_same_seeds():
    # the whole pipeline; the oracle refines the same refinement seeds with the
    # same kicks, and its winners must reach the targets about as often
    P = 16
    w, sol, tj, anc, tgt, _ = chain(P=P, S=8)
    g = torch.Generator(device=DEV).manual_seed(0)
    prev = t(w.model.random_cfgs(np.random.default_rng(9), P))
    best, score, parts = sol.solve(t(w.target_T), prev, num_seeds=32, coarse_max_iter=20, lm_max_iter=40,
                                   generator=g, return_all=True, **REF_KW)
    seeds, ccfg, cerr, lm_seeds, kicks, rcfg, rerr = (x.cpu().numpy() for x in parts)
    assert lm_seeds.shape == (P, 30, w.model.n_act) and kicks.shape == (P, 30, 40, w.model.n_act)
    # the winner is the refinement output of least error
    np.testing.assert_array_equal(best.cpu().numpy(), rcfg[np.arange(P), np.argmin(rerr, axis=1)])
    md = w.model.as_dict()
    ok_gpu, ok_or = [], []
    for p in range(P):
        ocfg, oerr, _ = ohjcd.lm_refine(lm_seeds[p], kicks[p], tgt[p:p + 1], md, tj, anc, w.model.lower,
                                        w.model.upper, np.zeros(w.model.n_act, bool), max_iter=40, stall_patience=6,
                                        eps_pos=1e-8, eps_ori=1e-8, **REF_KW)
        for cfg, acc in ((best.cpu().numpy()[p], ok_gpu), (ocfg[np.argmin(oerr)], ok_or)):
            pe, re = olm.pose_errors(cfg[None].astype(np.float64), w.target_T[p:p + 1], md, tj[0])
            acc.append(bool(pe[0] < 1e-3 and re[0] < 1e-2))
    assert np.mean(ok_gpu) >= 0.5
    assert abs(np.mean(ok_gpu) - np.mean(ok_or)) <= 0.15, (np.mean(ok_gpu), np.mean(ok_or))
    assert np.mean(np.asarray(ok_gpu) == np.asarray(ok_or)) >= 0.8


def test_refinement_over_two_seed_chunks_and_empty_batch():
    """45 refinement seeds: the block walks a chunk of 32 and one of 13; no problems at all."""
    w, sol, tj, anc, tgt, oc = chain(P=2, S=45, coll=True)
    noise = np.random.default_rng(11).normal(size=(2, 45, 6, w.model.n_act)).astype(np.float32)
    cfg, err, stop = sol.refine(t(w.seeds), t(noise), t(w.target_T), max_iter=6, **REF_KW)
    err = err.cpu().numpy()
    for p in range(2):
        _, oe, ostop = ohjcd.lm_refine(w.seeds[p], noise[p], tgt[p:p + 1], w.model.as_dict(), tj, anc,
                                       w.model.lower, w.model.upper, np.zeros(w.model.n_act, bool), max_iter=6,
                                       stall_patience=6, eps_pos=1e-8, eps_ori=1e-8, coll=oc, **REF_KW)
        assert agree(err[p], oe, rtol=1e-2, atol=1e-8) >= 0.85
        assert int(stop[p]) == int(ostop)
    c0, e0, s0 = sol.refine(t(w.seeds[:0]), t(noise[:0]), t(w.target_T[:0]), max_iter=6, **REF_KW)
    assert c0.shape == (0, 45, w.model.n_act) and s0.shape == (0,)
