"""The reference's JAX LM variant -- oracle (test infrastructure only).

Restates ``_ls_ik_single`` (``src/pyroffi/optimization_engines/_ls_ik.py:192-350``)
and the winner selection of ``ls_ik_solve`` (``:495-513``) in FP64 numpy,
vectorised over seeds.  It differs from the CUDA variant (``oracle/lm.py``)
in these points, each as the JAX code has it:

* the residual of each end effector is the body-frame SE(3) logarithm
  ``(T_actual^-1 @ T_target).log()`` in jaxlie's ``[v, omega]`` layout
  (``_ik_primitives.py:94-103``), not the world-frame position difference
  and the rotation vector of ``q_ee * conj(q_tgt)``;
* the Jacobian is the derivative of that residual (``jax.vjp`` there; here
  central differences in FP64 with step 1e-6, whose error, about 1e-10, is far
  below the FP32 effects the oracle is used to judge);
* the damped system is solved with a general solve (``jnp.linalg.solve``),
  not a Cholesky with a zero step on a non-positive pivot, and fixed joints
  are masked after the solve, not in the matrix;
* the trust radius reads the norms of the ``v`` and ``omega`` parts of the
  body-frame residual, max over end effectors;
* there is no convergence exit: every seed runs ``max_iter`` iterations;
* λ goes ×0.5 on accept and ×3 on reject, clipped to [1e-10, 1e6];
* collision and other constraints enter as extra residual rows
  ``sqrt(w_c) * c(q)`` (``:245-251``).  ``collision_constraint`` below builds
  the one that reproduces the CUDA variant's hinge² penalty, so that both
  variants minimise the same collision term.

Shared with the CUDA variant: weights ``[pos x3, ori x3]`` per end effector,
Jacobi column scale ``||J[:, a]|| + 1e-8``, trust radii 0.38 / 0.22 / 0.12 /
0.05 with their thresholds, the 5-point line search over clamped trials
(first minimum wins), accept at ``err < curr * (1 - 1e-4)``, all-time best
tracking.
"""

from __future__ import annotations

import numpy as np

from . import collision, kinematics, se3

ALPHAS = (1.0, 0.5, 0.25, 0.1, 0.025)
FD_STEP = 1e-6


def _fk(cfg, model):
    return kinematics.fk_joints(cfg, model["twists"], model["parent_tf"], model["parent_idx"],
                                model["act_idx"], model["mimic_mul"], model["mimic_off"],
                                model["mimic_act_idx"], model["topo_inv"])


def body_log_residual(T_joints, target_jnts, target_T):
    """[S, 6*n_ee]: per EE ``log(T_ee^-1 @ T_target)`` as ``[v, omega]``.

    T_joints [S, n_j, 7] (wxyz_xyz); target_T [S or 1, n_ee, 7]."""
    parts = []
    for e, tj in enumerate(target_jnts):
        Tee = T_joints[:, tj, :]
        tgt = np.broadcast_to(target_T[:, e, :], Tee.shape)
        parts.append(se3.log(se3.compose(se3.inverse(Tee), tgt)))
    return np.concatenate(parts, axis=-1)


def collision_constraint(model, spheres_local, sphere_joint, ws=None, self_i=None, self_j=None, margin=0.02):
    """c(q) = sqrt(sum of hinge² terms) [S]: with weight w_c, ``w_c * c²`` is the
    CUDA variant's penalty ``w_c * sum hinge²`` (``collision.lm_penalty``) on
    the same robot spheres, world spheres and sphere pairs, evaluated with
    sphere-only arithmetic (the world here holds spheres only)."""
    ws = np.zeros((0, 4)) if ws is None else np.asarray(ws, np.float64)
    sl = np.asarray(spheres_local, np.float64)
    sj = np.asarray(sphere_joint)
    valid = (sj >= 0) & (sj < model["n_joints"])
    r_all = sl[:, 3]
    si = None if self_i is None or len(self_i) == 0 else np.asarray(self_i)
    sjj = None if si is None else np.asarray(self_j)
    wo = np.ascontiguousarray(ws[:, :3])
    o2 = np.sum(wo * wo, axis=-1)
    rsum = r_all[valid][:, None] + ws[None, :, 3]                   # [n_valid, Ms]
    reach2 = np.where(rsum + margin > 0, (rsum + margin) ** 2 * (1 + 1e-9) + 1e-12, 0.0)

    def c(q):
        Tj = _fk(q, model)
        P = collision.robot_sphere_world(Tj, sl, np.where(valid, sj, 0))        # [S, n_rs, 3]
        pen = np.zeros(P.shape[0])
        if len(ws):
            Pv = P[:, valid]
            # |p - o|^2 = |p|^2 + |o|^2 - 2 p.o, the cross term as one matrix product
            d2 = np.sum(Pv * Pv, axis=-1)[..., None] + o2[None, None, :] - 2.0 * (Pv @ wo.T)
            # only pairs closer than r + r_o + margin have a non-zero hinge
            s_idx, k_idx, m_idx = np.nonzero(d2 < reach2[None])
            d = np.sqrt(np.maximum(d2[s_idx, k_idx, m_idx], 0.0)) - rsum[k_idx, m_idx]
            h = np.minimum(d - margin, 0.0)
            pen += np.bincount(s_idx, weights=h * h, minlength=P.shape[0])
        if si is not None:
            d = np.sqrt(np.sum((P[:, si] - P[:, sjj]) ** 2, axis=-1)) - (r_all[si] + r_all[sjj])
            h = np.minimum(d - margin, 0.0)
            pen += np.sum(h * h, axis=-1)
        return np.sqrt(pen)
    return c


def ls_ik_jax(seeds, target_T, model, target_jnts, *, lower, upper, fixed_mask=None, max_iter=60,
              pos_weight=50.0, ori_weight=10.0, lambda_init=5e-3, constraint=None, constraint_weight=0.0):
    """Each seed of ``seeds [S, n_act]`` refined against ``target_T [S or 1, n_ee, 7]``.

    Returns (best_cfg [S, n_act], best_err [S]) in FP64, ``best_err`` being
    the objective (weighted residual² plus constraint rows²) of ``best_cfg``.
    """
    c = np.array(seeds, dtype=np.float64)
    S, n = c.shape
    target_T = np.asarray(target_T, np.float64)
    if target_T.ndim == 2:
        target_T = target_T[None]
    lower = np.asarray(lower, np.float64)
    upper = np.asarray(upper, np.float64)
    fixed = np.zeros(n, bool) if fixed_mask is None else np.asarray(fixed_mask).astype(bool)
    n_ee = len(target_jnts)
    W = np.tile(np.array([pos_weight] * 3 + [ori_weight] * 3, np.float64), n_ee)
    sqrt_wc = np.sqrt(constraint_weight)

    def fused(q):
        f = body_log_residual(_fk(q, model), target_jnts, target_T) * W
        if constraint is not None:
            f = np.concatenate([f, (sqrt_wc * constraint(q))[:, None]], axis=-1)
        return f

    def err(q):
        f = fused(q)
        return np.sum(f * f, axis=-1)

    lam = np.full(S, lambda_init, np.float64)
    best_c = c.copy()
    best_err = err(c)
    for _ in range(max_iter):
        f = fused(c)
        curr = np.sum(f * f, axis=-1)
        J = np.empty((S, f.shape[1], n))
        for a in range(n):
            dq = np.zeros(n)
            dq[a] = FD_STEP
            J[:, :, a] = (fused(c + dq) - fused(c - dq)) / (2.0 * FD_STEP)
        col = np.linalg.norm(J, axis=1) + 1e-8
        Js = J / col[:, None, :]
        A = np.einsum("ska,skb->sab", Js, Js) + lam[:, None, None] * np.eye(n)
        rhs = -np.einsum("ska,sk->sa", Js, f)
        p = np.linalg.solve(A, rhs[..., None])[..., 0]
        delta = np.where(fixed[None, :], 0.0, p / col)
        max_p = np.zeros(S)
        max_o = np.zeros(S)
        for e in range(n_ee):
            max_p = np.maximum(max_p, np.linalg.norm(f[:, 6 * e:6 * e + 3] / W[:3], axis=-1))
            max_o = np.maximum(max_o, np.linalg.norm(f[:, 6 * e + 3:6 * e + 6] / W[3:6], axis=-1))
        R = np.where((max_p > 1e-2) | (max_o > 0.6), 0.38,
             np.where((max_p > 1e-3) | (max_o > 0.25), 0.22,
              np.where((max_p > 2e-4) | (max_o > 0.08), 0.12, 0.05)))
        dn = np.linalg.norm(delta, axis=-1) + 1e-18
        delta = np.where((dn > R)[:, None], delta * (R / dn)[:, None], delta)
        errs = np.stack([err(np.clip(c + a * delta, lower, upper)) for a in ALPHAS], axis=-1)
        bi = np.argmin(errs, axis=-1)
        new_err = errs[np.arange(S), bi]
        new_c = np.clip(c + np.asarray(ALPHAS)[bi][:, None] * delta, lower, upper)
        improved = new_err < curr * (1.0 - 1e-4)
        c = np.where(improved[:, None], new_c, c)
        lam = np.clip(np.where(improved, lam * 0.5, lam * 3.0), 1e-10, 1e6)
        better = new_err < best_err
        best_c = np.where(better[:, None], new_c, best_c)
        best_err = np.where(better, new_err, best_err)
    return best_c, best_err


def weighted_body_error(cfg, target_T, model, target_jnts, pos_weight=50.0, ori_weight=10.0):
    """The JAX variant's winner score without constraints: sum over EEs of
    ``||W * log(T_ee^-1 @ T_target)||²`` (``_ls_ik.py:502-508``), cfg [..., n_act]."""
    shp = cfg.shape[:-1]
    q = np.asarray(cfg, np.float64).reshape(-1, cfg.shape[-1])
    tT = np.asarray(target_T, np.float64)
    tT = np.broadcast_to(tT.reshape((-1,) + tT.shape[-2:]) if tT.ndim >= 3 else tT[None], (q.shape[0],) + tT.shape[-2:])
    f = body_log_residual(_fk(q, model), target_jnts, tT)
    W = np.tile(np.array([pos_weight] * 3 + [ori_weight] * 3, np.float64), len(target_jnts))
    return np.sum((f * W) ** 2, axis=-1).reshape(shp)


def select_winner(cfgs, errs):
    """argmin over seeds (``_ls_ik.py:511-513``); cfgs [P, S, n], errs [P, S]."""
    idx = np.argmin(errs, axis=-1)
    return cfgs[np.arange(cfgs.shape[0]), idx], idx
