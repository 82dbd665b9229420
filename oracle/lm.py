"""Multi-seed Levenberg-Marquardt IK -- oracle (test infrastructure only).

Restates ``ls_ik_lm_kernel`` (``src/pyroffi/cuda_kernels/_ls_ik_cuda_kernel.cu:65-394``)
step for step, vectorised over seeds with numpy:

* residual / stacked geometric Jacobian per end-effector
  (``compute_multi_ee_residual_and_jacobian``, ``_ik_cuda_helpers.cuh:433-551``):
  world-frame position difference and the rotation vector of
  ``q_ee * conj(q_tgt)`` (sign-folded to w >= 0, ``2 v`` below
  sin(theta/2) = 1e-6); Jacobian columns ``z x (p_ee - p_j)`` / ``z`` for
  revolute joints and ``z`` / 0 for prismatic ones, scaled by the mimic
  multiplier and restricted to each EE's ancestor joints;
* row weights ``[pos_weight x3, ori_weight x3]``, current error including the
  collision hinge penalty (``:166-229``, ``:258-267``);
* Jacobi column scaling ``||J[:,a]|| + 1e-8`` (``:270-279``);
* damped normal equations ``(Js^T Js + lam I) p = -Js^T fw`` with fixed-joint
  masking and a Cholesky solve that returns p = 0 on a non-positive pivot
  (``:282-307``, ``_ik_cuda_helpers.cuh:207-243``);
* trust-region radius from the max position / orientation error over EEs
  (``:315-335``);
* 5-point line search over alpha in {1, .5, .25, .1, .025} on clamped trial
  configurations (``:338-367``), first minimum wins;
* accept if ``err < curr * (1 - 1e-4)``: ``lam = max(lam*down, 1e-10)``, else
  ``lam = min(lam*up, 1e6)`` (reference factors down = 0.5, up = 3;
  ``:376-382``);
* all-time best tracking (``:385-388``) and the all-EE convergence exit
  (``:246-255``).

The optional explicit robot-sphere pair list adds a self-collision hinge to
the same penalty (an extension the reference kernel does not have).

``pose_errors`` restates ``_pose_errors`` of ``tests/bench_ik.py:341-353``.
"""

from __future__ import annotations

import numpy as np

from . import collision, kinematics, se3

ALPHAS = (1.0, 0.5, 0.25, 0.1, 0.025)


def residual_and_jacobian(T_joints, target_jnts, target_T, model, ancestor_masks, want_jac=True):
    """r [S, 6*n_ee] and J [S, 6*n_ee, n_act] for joint poses T_joints [S, n_j, 7].

    target_T: [S or 1, n_ee, 7].
    """
    S = T_joints.shape[0]
    n_ee = len(target_jnts)
    n_act = model["n_act"]
    r = np.zeros((S, 6 * n_ee), T_joints.dtype)
    J = np.zeros((S, 6 * n_ee, n_act), T_joints.dtype) if want_jac else None
    arms = []
    for e, tj in enumerate(target_jnts):
        Tee = T_joints[:, tj, :]
        tgt = np.broadcast_to(target_T[:, e, :], Tee.shape)
        r[:, 6 * e:6 * e + 3] = Tee[:, 4:7] - tgt[:, 4:7]
        qerr = se3.quat_mul(Tee[:, :4], se3.quat_conj(tgt[:, :4]))
        qerr = np.where(qerr[:, :1] < 0, -qerr, qerr)
        sh = np.linalg.norm(qerr[:, 1:4], axis=-1)
        big = sh > 1e-6
        theta = 2.0 * np.arctan2(sh, qerr[:, 0])
        fac = np.where(big, theta / np.where(big, sh, 1.0), 2.0)
        r[:, 6 * e + 3:6 * e + 6] = qerr[:, 1:4] * fac[:, None]
        arms.append(Tee[:, 4:7])
    if not want_jac:
        return r, None
    tw = np.asarray(model["twists"], T_joints.dtype)
    for j in range(model["n_joints"]):
        a1 = int(model["act_idx"][j])
        a2 = int(model["mimic_act_idx"][j])
        if a1 < 0 and a2 < 0:
            continue
        ang2 = float(np.sum(tw[j, 3:6] ** 2))
        lin2 = float(np.sum(tw[j, 0:3] ** 2))
        if ang2 > 1e-6:
            rev = True
            ax = tw[j, 3:6] / np.sqrt(ang2)
        elif lin2 > 1e-6:
            rev = False
            ax = tw[j, 0:3] / np.sqrt(lin2)
        else:
            continue
        z = se3.quat_rotate(T_joints[:, j, :4], np.broadcast_to(ax, (S, 3)))
        pj = T_joints[:, j, 4:7]
        s = float(model["mimic_mul"][j])
        for e in range(n_ee):
            if not ancestor_masks[e][j]:
                continue
            if rev:
                lin = np.cross(z, arms[e] - pj)
                ang = z
            else:
                lin = z
                ang = np.zeros_like(z)
            col = np.concatenate([lin, ang], axis=-1) * s
            for a in (a1, a2):
                if a >= 0:
                    J[:, 6 * e:6 * e + 6, a] += col
    return r, J


def chol_solve(A, b):
    """Batched Cholesky solve; rows with a non-positive pivot return 0."""
    S, n, _ = A.shape
    L = np.zeros_like(A)
    ok = np.ones(S, dtype=bool)
    for k in range(n):
        s = A[:, k, k] - np.sum(L[:, k, :k] ** 2, axis=-1)
        ok &= s > 0
        lkk = np.sqrt(np.where(s > 0, s, 1.0))
        L[:, k, k] = lkk
        for i in range(k + 1, n):
            t = A[:, i, k] - np.sum(L[:, i, :k] * L[:, k, :k], axis=-1)
            L[:, i, k] = t / lkk
    y = np.zeros_like(b)
    for i in range(n):
        y[:, i] = (b[:, i] - np.sum(L[:, i, :i] * y[:, :i], axis=-1)) / L[:, i, i]
    x = np.zeros_like(b)
    for i in range(n - 1, -1, -1):
        x[:, i] = (y[:, i] - np.sum(L[:, i + 1:, i] * x[:, i + 1:], axis=-1)) / L[:, i, i]
    return np.where(ok[:, None], x, 0.0)


def _fk(cfg, model):
    return kinematics.fk_joints(cfg, model["twists"], model["parent_tf"], model["parent_idx"],
                                model["act_idx"], model["mimic_mul"], model["mimic_off"],
                                model["mimic_act_idx"], model["topo_inv"])


def ls_ik(seeds, target_T, model, target_jnts, ancestor_masks, *, lower, upper,
          fixed_mask=None, max_iter=30, pos_weight=50.0, ori_weight=10.0, lambda_init=5e-3,
          eps_pos=1e-8, eps_ori=1e-8, enable_collision=False, collision_weight=0.0,
          collision_margin=0.02, spheres_local=None, sphere_joint=None,
          ws=None, wc=None, wb=None, wh=None, self_i=None, self_j=None,
          lambda_down=0.5, lambda_up=3.0):
    """Run the LM for seeds [S, n_act] against target_T [S or 1, n_ee, 7].

    Returns (best_cfg [S, n_act], best_err [S]), FP64.
    """
    cfg = np.array(seeds, dtype=np.float64)
    S, n_act = cfg.shape
    target_T = np.asarray(target_T, np.float64)
    if target_T.ndim == 2:
        target_T = target_T[None]
    lower = np.asarray(lower, np.float64)
    upper = np.asarray(upper, np.float64)
    fixed = np.zeros(n_act, bool) if fixed_mask is None else np.asarray(fixed_mask).astype(bool)
    n_ee = len(target_jnts)
    W = np.tile(np.array([pos_weight] * 3 + [ori_weight] * 3, np.float64), n_ee)
    empty = {4: np.zeros((0, 4)), 7: np.zeros((0, 7)), 15: np.zeros((0, 15)), 6: np.zeros((0, 6))}
    ws = empty[4] if ws is None else np.asarray(ws, np.float64)
    wc = empty[7] if wc is None else np.asarray(wc, np.float64)
    wb = empty[15] if wb is None else np.asarray(wb, np.float64)
    wh = empty[6] if wh is None else np.asarray(wh, np.float64)
    use_coll = bool(enable_collision) and spheres_local is not None and len(spheres_local) > 0

    def penalty(Tj):
        if not use_coll:
            return np.zeros(Tj.shape[0])
        return collision.lm_penalty(Tj, spheres_local, sphere_joint, ws, wc, wb, wh,
                                    collision_margin, collision_weight, self_i, self_j)

    def err_of(c):
        Tj = _fk(c, model)
        r, _ = residual_and_jacobian(Tj, target_jnts, target_T, model, ancestor_masks, want_jac=False)
        return np.sum((r * W) ** 2, axis=-1) + penalty(Tj)

    best_cfg = cfg.copy()
    best_err = err_of(cfg)
    lam = np.full(S, lambda_init, np.float64)
    active = np.ones(S, dtype=bool)

    for _ in range(max_iter):
        Tj = _fk(cfg, model)
        r, J = residual_and_jacobian(Tj, target_jnts, target_T, model, ancestor_masks)
        conv = np.ones(S, dtype=bool)
        for e in range(n_ee):
            conv &= np.linalg.norm(r[:, 6 * e:6 * e + 3], axis=-1) < eps_pos
            conv &= np.linalg.norm(r[:, 6 * e + 3:6 * e + 6], axis=-1) < eps_ori
        active &= ~conv
        if not active.any():
            break
        fw = r * W
        Jw = J * W[None, :, None]
        curr = np.sum(fw * fw, axis=-1) + penalty(Tj)
        col = np.sqrt(np.sum(Jw * Jw, axis=1)) + 1e-8
        Js = Jw / col[:, None, :]
        A = np.einsum("ska,skb->sab", Js, Js) + lam[:, None, None] * np.eye(n_act)
        rhs = -np.einsum("ska,sk->sa", Js, fw)
        for a in np.nonzero(fixed)[0]:
            A[:, a, :] = 0.0
            A[:, :, a] = 0.0
            A[:, a, a] = 1.0
            rhs[:, a] = 0.0
        p = chol_solve(A, rhs)
        delta = p / col
        max_p = np.zeros(S)
        max_o = np.zeros(S)
        for e in range(n_ee):
            max_p = np.maximum(max_p, np.linalg.norm(r[:, 6 * e:6 * e + 3], axis=-1))
            max_o = np.maximum(max_o, np.linalg.norm(r[:, 6 * e + 3:6 * e + 6], axis=-1))
        R = np.where((max_p > 1e-2) | (max_o > 0.6), 0.38,
             np.where((max_p > 1e-3) | (max_o > 0.25), 0.22,
              np.where((max_p > 2e-4) | (max_o > 0.08), 0.12, 0.05)))
        dn = np.linalg.norm(delta, axis=-1)
        delta = np.where((dn > R)[:, None], delta * (R / (dn + 1e-18))[:, None], delta)
        errs = np.stack([err_of(np.clip(cfg + a * delta, lower, upper)) for a in ALPHAS], axis=-1)
        bi = np.argmin(errs, axis=-1)
        berr = errs[np.arange(S), bi]
        trial = np.clip(cfg + np.asarray(ALPHAS)[bi][:, None] * delta, lower, upper)
        improved = berr < curr * (1.0 - 1e-4)
        upd = active & improved
        cfg = np.where(upd[:, None], trial, cfg)
        lam = np.where(active, np.where(improved, np.maximum(lam * lambda_down, 1e-10),
                                        np.minimum(lam * lambda_up, 1e6)), lam)
        better = active & (berr < best_err)
        best_err = np.where(better, berr, best_err)
        best_cfg = np.where(better[:, None], trial, best_cfg)
    return best_cfg, best_err


def pose_errors(cfg, target_T, model, target_joint):
    """FP64 (position error [m], rotation error [rad]) of ``tests/bench_ik.py``'s
    ``_pose_errors``: ||t - t_tgt|| and ||log(R_tgt^-1 R)||."""
    Tj = _fk(cfg, model)
    T = Tj[..., target_joint, :]
    target_T = np.asarray(target_T, np.float64)
    pos = np.linalg.norm(T[..., 4:7] - target_T[..., 4:7], axis=-1)
    rel = se3.quat_mul(se3.quat_conj(target_T[..., :4]), T[..., :4])
    return pos, se3.rotation_angle(rel)


def select_winner(cfgs, errs, prev=None, continuity_weight=0.0):
    """argmin over seeds of err + w * ||q - prev||^2 (``_ls_ik.py:974-999``)."""
    score = np.asarray(errs, np.float64)
    if prev is not None and continuity_weight:
        score = score + continuity_weight * np.sum((cfgs - prev[:, None, :]) ** 2, axis=-1)
    idx = np.argmin(score, axis=-1)
    return cfgs[np.arange(cfgs.shape[0]), idx], idx
