"""GPU parity of the warp-per-seed LM body and of the persistent batched IK.

* The warp body (wide robots: 15-DOF bimanual tree, 29-DOF humanoid, two
  hand targets; and the 7-DOF chain when forced) against the FP64 oracle,
  seed by seed over a few iterations (FP32 vs FP64 accept decisions may part
  on a few seeds, as for the seed-group kernel).
* The persistent batch (``pk_ik_batch``, mixed classes, uneven seed counts)
  against the per-class launches on the same padded buffers: the same
  device code runs per seed, so the results are identical.
* CUDA-graph replay of the batch equals the eager run.
"""

import numpy as np
import pytest
import torch

from oracle import lm as olm
from pyroffi_b200 import workloads as W
from pyroffi_b200.batch_ik import BODY_SEED_GROUP, BODY_SEED_GROUP16, BODY_WARP, MixedIkBatch
from pyroffi_b200.ik import BatchIkSolver

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def tt(x):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float32, device=DEV)


def opts(w, **kw):
    o = dict(max_iter=w.max_iter, lambda_init=w.lambda_init, lambda_down=w.lambda_down, lambda_up=w.lambda_up,
             collision_weight=w.collision_weight, collision_margin=w.collision_margin, pos_tol=w.pos_tol,
             rot_tol=w.rot_tol)
    o.update(kw)
    return o


@pytest.fixture(scope="module")
def mixed():
    return W.mixed_ik(n_problems=48, seeds_range=(8, 40))


def class_oracle(w, c, p, seeds, max_iter):
    cl = w.classes[c]
    m = cl.model
    rs, jidx, _ = cl.spheres.flat_for_ik(m)
    return olm.ls_ik(seeds, w.target_T[c][p][None], m.as_dict(), [m.link_joint(l) for l in cl.target_links],
                     [m.ancestor_mask(l) for l in cl.target_links], lower=m.lower, upper=m.upper,
                     max_iter=max_iter, lambda_init=w.lambda_init, lambda_down=w.lambda_down,
                     lambda_up=w.lambda_up, enable_collision=True, collision_weight=w.collision_weight,
                     collision_margin=w.collision_margin, spheres_local=rs, sphere_joint=jidx,
                     ws=w.world.spheres)


@pytest.mark.parametrize("c,tps", [(3, 0), (3, 32), (2, 16), (2, 32), (0, 16)])
@pytest.mark.parametrize("max_iter", [0, 1, 2])
def test_warp_body_few_iterations_vs_oracle(mixed, c, tps, max_iter):
    w = mixed
    cl = w.classes[c]
    s = BatchIkSolver(cl.model, cl.target_links, spheres=cl.spheres, world=w.world, device=DEV,
                      **opts(w, max_iter=max_iter, threads_per_seed=tps))
    P = 3
    seeds = w.seeds[c][:P, :16]
    cfgs, errs = s.run_lm(tt(w.target_T[c][:P]), tt(seeds))
    cfgs, errs = cfgs.cpu().numpy(), errs.cpu().numpy()
    ok = 0
    for p in range(P):
        oc, oe = class_oracle(w, c, p, seeds[p], max_iter)
        close = (np.abs(cfgs[p] - oc).max(axis=1) < 2e-4) & (np.abs(errs[p] - oe) <= 1e-3 * np.abs(oe) + 1e-4)
        ok += int(close.sum())
    assert ok >= 0.9 * P * 16, ok


def test_warp_body_initial_error(mixed):
    w = mixed
    c = 3
    cl = w.classes[c]
    s = BatchIkSolver(cl.model, cl.target_links, spheres=cl.spheres, world=w.world, device=DEV, **opts(w, max_iter=0))
    seeds = w.seeds[c][:2, :24]
    cfgs, errs = s.run_lm(tt(w.target_T[c][:2]), tt(seeds))
    np.testing.assert_array_equal(cfgs.cpu().numpy(), seeds)
    for p in range(2):
        _, oe = class_oracle(w, c, p, seeds[p], 0)
        np.testing.assert_allclose(errs[p].cpu().numpy(), oe, rtol=2e-5, atol=1e-5)


def per_class_reference(w, b):
    """Per-class launches on the batch's own padded buffers."""
    out = []
    for c, cl in enumerate(w.classes):
        if b.counts[c] == 0:
            out.append(None)
            continue
        # the same mappings as the batch's bodies: one lane per seed (bodies 0 and 2), the warp body (1)
        tps = {BODY_SEED_GROUP: 1, BODY_SEED_GROUP16: 0, BODY_WARP: 16}[b.bodies[c]]
        s = BatchIkSolver(cl.model, cl.target_links, spheres=cl.spheres, world=w.world, device=DEV,
                          **opts(w, threads_per_seed=tps))
        # the batch's grid resolution, named (the default one is fitted to each launch's shared memory)
        s.opt.obstacle_grid = b.opt.obstacle_grid
        out.append(s.run_lm(b.targets[c], b.seeds[c]))
    return out


def used_mask(b, c):
    m = np.zeros((b.counts[c], b.strides[c]), bool)
    for p in np.nonzero(b.problem_class == c)[0]:
        m[b.index_in_class[p], : b.n_seeds[p]] = True
    return m


def make_batch(w, **kw):
    b = MixedIkBatch(w.classes, w.world, device=DEV, **opts(w, **kw))
    b.prepare(w.problem_class, w.n_seeds)
    b.load(w.target_T, w.seeds)
    return b


def test_batch_equals_per_class_launches(mixed):
    w = mixed
    b = make_batch(w)
    b.opt.obstacle_grid = 12
    assert b.bodies == [BODY_SEED_GROUP, BODY_SEED_GROUP, BODY_SEED_GROUP16, BODY_WARP]
    b.run_lm()
    ref = per_class_reference(w, b)
    for c in range(len(w.classes)):
        if b.counts[c] == 0:
            continue
        m = used_mask(b, c)
        np.testing.assert_array_equal(b.out_cfg[c].cpu().numpy()[m], ref[c][0].cpu().numpy()[m])
        np.testing.assert_array_equal(b.out_err[c].cpu().numpy()[m], ref[c][1].cpu().numpy()[m])
        assert np.all(np.isinf(b.out_err[c].cpu().numpy()[~m]))


def test_batch_graph_replay_and_reload(mixed):
    w = mixed
    b = make_batch(w)
    eager = [r.winner_cfg.clone() if r is not None else None for r in b.solve()]
    b.capture()
    rep = b.solve()
    for c in range(len(w.classes)):
        if eager[c] is not None:
            torch.testing.assert_close(rep[c].winner_cfg, eager[c], rtol=0, atol=0)
    # new seeds through the same graph
    rng = np.random.default_rng(9)
    seeds2 = [rng.uniform(cl.model.lower, cl.model.upper, size=s.shape).astype(np.float32)
              for cl, s in zip(w.classes, w.seeds)]
    b.load(w.target_T, seeds2)
    rep2 = [r.winner_cfg.clone() if r is not None else None for r in b.solve()]
    b2 = make_batch(w)
    b2.load(w.target_T, seeds2)
    eager2 = b2.solve()
    for c in range(len(w.classes)):
        if rep2[c] is not None:
            torch.testing.assert_close(rep2[c], eager2[c].winner_cfg, rtol=0, atol=0)


def test_batch_autotune_keeps_results(mixed):
    w = mixed
    b = make_batch(w)
    b.run_lm()
    base = [e.clone() for e in b.out_err]
    res = b.autotune(candidates=((2, 64), (4, 32)), wide_lanes=(16, 32), grids=(0, -1), reps=1)
    assert set(res) == {(t, s, l, g) for t, s in ((2, 64), (4, 32)) for l in (16, 32) for g in (0, -1)}
    b.run_lm()
    # lanes per seed change the order of the penalty sum only; an accept test
    # on the edge may flip for a few seeds
    for c in range(len(w.classes)):
        m = torch.as_tensor(used_mask(b, c), device=DEV)
        a, e = b.out_err[c][m].cpu().numpy(), base[c][m].cpu().numpy()
        assert np.mean(np.abs(a - e) <= 1e-4 * np.abs(e) + 1e-5) >= 0.95


def test_batch_success_vs_oracle_small(mixed):
    """Full 30-iteration solves of 2 problems per class: GPU success >= oracle's - 1 per class."""
    w = mixed
    b = make_batch(w)
    res = b.solve()
    for c, cl in enumerate(w.classes):
        if b.counts[c] == 0:
            continue
        probs = np.nonzero(w.problem_class == c)[0][:2]
        or_ok = 0
        for p in probs:
            i = int(w.index_in_class[p])
            seeds = w.seeds[c][i, : w.n_seeds[p]]
            oc, oe = class_oracle(w, c, i, seeds, w.max_iter)
            win = oc[np.argmin(oe)]
            m = cl.model
            pe_all, re_all = [], []
            for e, l in enumerate(cl.target_links):
                pe, re = olm.pose_errors(win[None].astype(np.float64), w.target_T[c][i][e][None].astype(np.float64),
                                         m.as_dict(), m.link_joint(l))
                pe_all.append(pe[0]); re_all.append(re[0])
            or_ok += int(max(pe_all) < w.pos_tol and max(re_all) < w.rot_tol)
        gpu_ok = int(res[c].success.cpu().numpy()[[int(w.index_in_class[p]) for p in probs]].sum())
        assert gpu_ok >= or_ok - 1, (c, gpu_ok, or_ok)


@pytest.mark.parametrize("grid", [4, 12, 16, -1])
def test_obstacle_tile_leaves_results_unchanged(mixed, grid):
    """The obstacle tile (cells per axis of the per-block grid, or none) only
    changes which obstacles take the bounding test.  The seed-group bodies
    still sum the hinge terms of each joint in increasing obstacle order, so
    their outputs are the same bits as with the default grid; the warp body
    spreads the (joint, candidate) pairs over its lanes by list position, so
    its sums may change order (rounding only)."""
    w = mixed
    b = make_batch(w)
    b.run_lm()
    base = [(c.clone(), e.clone()) for c, e in zip(b.out_cfg, b.out_err)]
    b.opt.obstacle_grid = grid
    b.run_lm()
    for c in range(len(w.classes)):
        m = torch.as_tensor(used_mask(b, c), device=DEV)
        if b.bodies[c] != BODY_WARP:
            assert torch.equal(b.out_err[c][m], base[c][1][m]), c
            assert torch.equal(b.out_cfg[c][m], base[c][0][m]), c
        else:
            a, e = b.out_err[c][m].cpu().numpy(), base[c][1][m].cpu().numpy()
            assert np.mean(np.abs(a - e) <= 1e-4 * np.abs(e) + 1e-5) >= 0.95
