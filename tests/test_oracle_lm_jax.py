"""The oracle's restatement of the reference's JAX LM variant (body-frame
SE(3)-log residual, general solve).  Its SE(3) logarithm is pinned to the
reference helpers' golden exponentials by a round trip; its collision rows
reproduce the CUDA variant's hinge² penalty; a small solve converges."""

import numpy as np

from oracle import collision as oc
from oracle import lm as olm
from oracle import lm_jax as oj
from oracle import se3
from pyroffi_b200 import workloads as W


def test_se3_log_inverts_reference_exp(golden):
    """log(exp(xi)) == xi on the reference helper's own exponentials.  The
    first 32 golden tangents are revolute / prismatic motions (exact in the
    reference); rotation angles stay below pi, where log is single-valued."""
    tang = golden["se3_exp_in"].astype(np.float64)[:32]
    T = golden["se3_exp_out"].astype(np.float64)[:32]
    T[:, :4] /= np.linalg.norm(T[:, :4], axis=-1, keepdims=True)
    assert np.all(np.linalg.norm(tang[:, 3:], axis=-1) < np.pi)
    np.testing.assert_allclose(se3.log(T), tang, atol=2e-6, rtol=1e-5)


def test_body_log_residual_zero_at_target_and_frame():
    w = W.ik(P=4, Sd=8)
    md = w.model.as_dict()
    tj = [w.model.link_joint(w.target_link)]
    Tj = oj._fk(w.target_cfgs.astype(np.float64), md)
    r = oj.body_log_residual(Tj, tj, w.target_T[:, None].astype(np.float64))
    assert np.abs(r).max() < 1e-6          # the targets are FK of target_cfgs (FP32-stored)
    # a pure world translation d of the target shows up as R_ee^T d in the v part
    d = np.array([0.01, -0.02, 0.005])
    tgt = Tj[:, tj[0]].copy()
    tgt[:, 4:7] += d
    r2 = oj.body_log_residual(Tj, tj, tgt[:, None])
    expect = se3.quat_rotate(se3.quat_conj(Tj[:, tj[0], :4]), np.broadcast_to(d, (4, 3)))
    np.testing.assert_allclose(r2[:, :3], expect, atol=1e-12)
    np.testing.assert_allclose(r2[:, 3:], 0.0, atol=1e-12)


def test_collision_rows_reproduce_the_cuda_penalty():
    w = W.ik(P=2, Sd=16)
    md = w.model.as_dict()
    q = w.seeds[0].astype(np.float64)
    c = oj.collision_constraint(md, w.spheres_local, w.sphere_joint, w.world.spheres, w.self_pairs[:, 0],
                                w.self_pairs[:, 1], w.collision_margin)
    pen = oc.lm_penalty(olm._fk(q, md), w.spheres_local, w.sphere_joint, w.world.spheres, np.zeros((0, 7)),
                        np.zeros((0, 15)), np.zeros((0, 6)), w.collision_margin, w.collision_weight,
                        w.self_pairs[:, 0], w.self_pairs[:, 1])
    np.testing.assert_allclose(w.collision_weight * c(q) ** 2, pen, rtol=1e-12, atol=1e-12)
    assert (pen > 0).any()


def test_jax_variant_solves_and_tracks_best():
    w = W.ik(P=2, Sd=32)
    md = w.model.as_dict()
    tj = [w.model.link_joint(w.target_link)]
    for p in range(2):
        e0 = oj.weighted_body_error(w.seeds[p], w.target_T[p][None, None], md, tj)
        cfg, err = oj.ls_ik_jax(w.seeds[p], w.target_T[p][None, None], md, tj, lower=w.model.lower,
                                upper=w.model.upper, max_iter=30, lambda_init=w.lambda_init)
        np.testing.assert_allclose(err, oj.weighted_body_error(cfg, w.target_T[p][None, None], md, tj),
                                   rtol=1e-9, atol=1e-15)
        assert np.all(err <= e0 + 1e-15)
        win, _ = oj.select_winner(cfg[None], err[None])
        pe, re = olm.pose_errors(win, w.target_T[p][None], md, tj[0])
        assert pe[0] < 1e-3 and re[0] < 1e-2, (pe, re)
        assert np.all(cfg >= w.model.lower - 1e-12) and np.all(cfg <= w.model.upper + 1e-12)
