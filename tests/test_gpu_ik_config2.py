"""The headline IK workload at full size, run exactly as the benchmark runs it
(256 targets x 128 seeds x 30 LM iterations, 7-DOF chain, 100 obstacle
spheres + 200 self pairs, margin 0.02, damping 1e-2 x0.1 / x10, FP64
verification at 1 mm / 0.01 rad), against

* the C port of the reference LM loop (``oracle/cpu``: FP32 with FP64
  normal equations, as the reference kernel) on the same 256 problems and
  seeds: seed-by-seed weighted errors, per-problem best errors and
  per-problem success;
* the FP64 restatement of the reference's JAX LM variant (body-frame SE(3)
  log residual, general solve; ``oracle/lm_jax.py``) on a sample of
  problems: the success of its winners and their final residuals next to
  the GPU's.

The measured figures go to the error report (``error_report``)."""

import numpy as np
import pytest
import torch

from error_report import record
from oracle import cpu_port
from oracle import lm as olm
from oracle import lm_jax as oj
from pyroffi_b200 import workloads as W
from pyroffi_b200.ik import BatchIkSolver

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


@pytest.fixture(scope="module")
def config2():
    w = W.ik(P=256, Sd=128, seed=1002)
    s = BatchIkSolver(w.model, w.target_link, spheres=w.spheres, world=w.world, self_pairs=w.self_pairs,
                      max_iter=w.max_iter, lambda_init=w.lambda_init, lambda_down=w.lambda_down,
                      lambda_up=w.lambda_up, pos_weight=w.pos_weight, ori_weight=w.ori_weight,
                      collision_weight=w.collision_weight, collision_margin=w.collision_margin,
                      pos_tol=w.pos_tol, rot_tol=w.rot_tol, device=DEV)
    r = s.solve(torch.as_tensor(w.target_T, device=DEV), torch.as_tensor(w.seeds, device=DEV))
    torch.cuda.synchronize()
    return w, r


def test_workload_is_the_benchmark_workload(config2):
    w, _ = config2
    assert w.seeds.shape == (256, 128, 7) and w.max_iter == 30
    assert len(w.world.spheres) == 100 and len(w.self_pairs) == 200
    assert (w.lambda_init, w.lambda_down, w.lambda_up, w.collision_margin) == (1e-2, 0.1, 10.0, 0.02)


def test_config2_against_the_port_on_all_problems(config2):
    w, r = config2
    lib = cpu_port.load()
    _, cfg_c, err_c = cpu_port.ls_ik(lib, w, 0, 256, cpu_port.max_threads(lib))
    err_g = r.errs.cpu().numpy()
    # seed by seed: the same weighted error (FP32 on both sides, different
    # operation order; accept / reject decisions on the edge may flip)
    seed_ok = np.abs(err_g - err_c) <= 1e-3 * np.abs(err_c) + 1e-6
    record("IK seed agreement with the C port (fraction of 32,768 seeds that differ)", 1.0 - seed_ok.mean(),
           "256 x 128 x 30")
    assert seed_ok.mean() >= 0.95, seed_ok.mean()
    # per problem: the best weighted error found
    bg, bc = err_g.min(axis=1), err_c.min(axis=1)
    prob_ok = np.abs(bg - bc) <= 1e-3 * np.abs(bc) + 1e-6
    assert prob_ok.mean() >= 0.95, prob_ok.mean()
    # success on the same problems, FP64-verified on both sides
    succ_c = cpu_port.success(w, 0, cfg_c, err_c)
    succ_g = r.success.cpu().numpy().astype(bool)
    assert succ_g.sum() >= succ_c.sum(), (int(succ_g.sum()), int(succ_c.sum()))
    assert (succ_g == succ_c).mean() >= 0.95
    # the kernel's FP32 weighted error of each winner against its FP64 recomputation
    win = r.winner_cfg.cpu().numpy().astype(np.float64)
    md = w.model.as_dict()
    tj = w.model.link_joint(w.target_link)
    Tj = olm._fk(win, md)
    res, _ = olm.residual_and_jacobian(Tj, [tj], w.target_T[:, None].astype(np.float64), md,
                                       [w.model.ancestor_mask(w.target_link)], want_jac=False)
    Wt = np.array([w.pos_weight] * 3 + [w.ori_weight] * 3)
    from oracle import collision as ocoll
    pen = ocoll.lm_penalty(Tj, w.spheres_local, w.sphere_joint, w.world.spheres, np.zeros((0, 7)),
                           np.zeros((0, 15)), np.zeros((0, 6)), w.collision_margin, w.collision_weight,
                           w.self_pairs[:, 0], w.self_pairs[:, 1])
    e64 = np.sum((res * Wt) ** 2, axis=-1) + pen
    e32 = err_g[np.arange(256), np.argmin(err_g, axis=1)]
    # Each term of the weighted error is (w * r)^2 with w = 50 for position,
    # 10 for rotation and sqrt(1e4) = 100 for a hinge of the collision
    # penalty; r comes from FP32 poses and sphere centres good to about 1e-6 m
    # (the measured FK and centre errors), so e carries an absolute error of
    # about 2 * sqrt(e) * 100 * 1e-6 on top of the FP32 relative rounding of
    # the sums.
    diff = np.abs(e32 - e64)
    rel = diff / np.maximum(np.abs(e64), 1e-12)
    big = e64 > 1e-2
    record("IK weighted error of the winner, FP32 kernel vs FP64 (relative, errors > 1e-2)", rel[big],
           "256 x 128 x 30")
    record("IK weighted error of the winner, FP32 kernel vs FP64 (absolute, errors <= 1e-2)", diff[~big],
           "256 x 128 x 30")
    assert np.all(diff <= 1e-4 * e64 + 2e-4 * np.sqrt(e64) + 1e-9), float(np.max(diff - 1e-4 * e64))
    record("IK final position error of solved problems (FP64)", r.pos_err.cpu().numpy()[succ_g], "256 x 128 x 30",
           "m")
    record("IK final rotation error of solved problems (FP64)", r.rot_err.cpu().numpy()[succ_g], "256 x 128 x 30",
           "rad")


def test_config2_against_the_jax_variant_on_a_sample(config2):
    """The JAX variant minimises the body-frame SE(3)-log residual (plus the
    same collision hinge², as constraint rows) with x0.5 / x3 damping.  On
    problems 0-3 its winners' success and final residuals are stated next to
    the GPU's; the GPU solves at least as many of them, minus one."""
    w, r = config2
    md = w.model.as_dict()
    tj = [w.model.link_joint(w.target_link)]
    con = oj.collision_constraint(md, w.spheres_local, w.sphere_joint, w.world.spheres, w.self_pairs[:, 0],
                                  w.self_pairs[:, 1], w.collision_margin)
    P = 4
    ok_j = np.zeros(P, bool)
    body_j, body_g = np.zeros(P), np.zeros(P)
    for p in range(P):
        cfg, err = oj.ls_ik_jax(w.seeds[p], w.target_T[p][None, None], md, tj, lower=w.model.lower,
                                upper=w.model.upper, max_iter=w.max_iter, lambda_init=w.lambda_init,
                                pos_weight=w.pos_weight, ori_weight=w.ori_weight, constraint=con,
                                constraint_weight=w.collision_weight)
        win, _ = oj.select_winner(cfg[None], err[None])
        pe, re = olm.pose_errors(win, w.target_T[p][None].astype(np.float64), md, tj[0])
        ok_j[p] = pe[0] < w.pos_tol and re[0] < w.rot_tol
        body_j[p] = np.sqrt(oj.weighted_body_error(win[0], w.target_T[p][None, None], md, tj))
        gw = r.winner_cfg[p].cpu().numpy().astype(np.float64)
        body_g[p] = np.sqrt(oj.weighted_body_error(gw, w.target_T[p][None, None], md, tj))
    ok_g = r.success.cpu().numpy()[:P].astype(bool)
    record("IK body-frame log residual ||W log(T^-1 T_tgt)|| of the GPU winner, problems 0-3", body_g,
           "256 x 128 x 30")
    record("IK body-frame log residual ||W log(T^-1 T_tgt)|| of the JAX-variant winner, problems 0-3", body_j,
           "same seeds, FP64")
    record("IK success on problems 0-3: GPU minus JAX variant", float(ok_g.sum() - ok_j.sum()), "")
    assert ok_g.sum() >= ok_j.sum() - 1, (ok_g, ok_j)
