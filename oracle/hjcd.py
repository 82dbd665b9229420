"""HJCD-IK -- FP64 oracle (test infrastructure only).

Restates the two kernels of the reference's CUDA HJCD-IK, vectorised over
the seeds of one problem with numpy:

* ``coarse`` -- ``hjcd_ik_coarse_kernel``
  (``src/pyroffi/cuda_kernels/_hjcd_ik_cuda_kernel.cu:91-321``): ``k_max``
  greedy coordinate-descent steps. Each step:
  - stacked residual / Jacobian (``oracle.lm.residual_and_jacobian``);
  - row weights 1 / ``clip((|r_p| + 1e-8) / (|r_o| + 1e-8), 0.05, 1)``, the
    orientation rows zeroed while ``|r_p| >= 1e-3`` (``adaptive_weights``,
    ``:53-66``);
  - the free joint with the largest ``(J_a^T f)^2 / (|J_a|^2 + 1e-8)`` (first
    maximum) takes ``-J_a^T f / (|J_a|^2 + 1e-8)``, clamped.

  The score is the unweighted squared error plus the hinge penalty
  (``oracle.collision.lm_penalty``).
* ``lm_refine`` -- ``hjcd_ik_lm_kernel`` (``:324-695``): adaptive row weights
  without gating, Jacobi column scaling, damped normal equations with the
  joint-limit prior ``lpw / h^2`` (``h = (upper - lower) / 2 + 1e-8``,
  gradient ``lpw / h^2 (q - mid)``), fixed joints masked, Cholesky (zero
  step on a non-positive pivot), trust region, a 5-point line search on the
  unweighted error that ends at the first new minimum with sufficient
  decrease, accept / reject (lambda x0.5 / x3 within [1e-10, 1e6]),
  all-time best, kicks ``noise[s, it] * kick_scale`` after ``stall_patience``
  rejections, and the problem-wide stop once a seed meets (eps_pos, eps_ori):
  every seed stops at the next iteration.

Parity is pinned through the components the golden vectors fix (FK,
residual / Jacobian, Cholesky, distances); the HJCD loop has no reference
output here (its kernels need XLA FFI to run).
"""

from __future__ import annotations

import numpy as np

from . import collision
from . import lm as olm

ALPHAS = (1.0, 0.5, 0.25, 0.1, 0.025)


def _penalty(Tj, coll):
    if coll is None:
        return np.zeros(Tj.shape[0])
    ws, wc, wb, wh = coll["world"]
    return collision.lm_penalty(Tj, coll["spheres_local"], coll["sphere_joint"], ws, wc, wb, wh, coll["margin"],
                                coll["weight"])


def _ee_norms(r, n_ee):
    rr = r.reshape(r.shape[0], n_ee, 6)
    return np.linalg.norm(rr[..., :3], axis=-1), np.linalg.norm(rr[..., 3:], axis=-1)   # [S, n_ee]


def _row_weights(r, n_ee, gate):
    pn, on = _ee_norms(r, n_ee)
    wo = np.clip((pn + 1e-8) / (on + 1e-8), 0.05, 1.0)
    if gate:
        wo = np.where(pn >= 1e-3, 0.0, wo)
    w = np.ones((r.shape[0], n_ee, 6))
    w[..., 3:] = wo[..., None]
    return w.reshape(r.shape[0], 6 * n_ee)


def coarse(seeds, target_T, model, target_jnts, anc, lower, upper, fixed, k_max, coll=None):
    """-> (cfg [S, n], err [S])."""
    cfg = np.array(seeds, np.float64)
    n_ee = len(target_jnts)
    free = ~np.asarray(fixed, bool)
    for _ in range(k_max):
        if not free.any():
            break
        Tj = olm._fk(cfg, model)
        r, J = olm.residual_and_jacobian(Tj, target_jnts, target_T, model, anc)
        w = _row_weights(r, n_ee, gate=True)
        fw = r * w
        Jw = J * w[:, :, None]
        dot = np.einsum("ska,sk->sa", Jw, fw)
        sq = np.sum(Jw * Jw, axis=1) + 1e-8
        impr = np.where(free[None, :], dot * dot / sq, -np.inf)
        best = np.argmax(impr, axis=1)
        idx = np.arange(cfg.shape[0])
        step = -dot[idx, best] / sq[idx, best]
        cfg[idx, best] = np.clip(cfg[idx, best] + step, lower[best], upper[best])
    Tj = olm._fk(cfg, model)
    r, _ = olm.residual_and_jacobian(Tj, target_jnts, target_T, model, anc, want_jac=False)
    return cfg, np.sum(r * r, axis=1) + _penalty(Tj, coll)


def _direction(r, J, cfg, lam, lower, upper, fixed, lpw, n_ee):
    w = _row_weights(r, n_ee, gate=False)
    fw = r * w
    Jw = J * w[:, :, None]
    cs = np.sqrt(np.sum(Jw * Jw, axis=1)) + 1e-8                       # [S, n]
    Js = Jw / cs[:, None, :]
    A = np.einsum("ski,skj->sij", Js, Js)
    rb = np.einsum("ski,sk->si", Js, fw)
    h = (upper - lower) * 0.5 + 1e-8
    mid = (lower + upper) * 0.5
    dpr = lpw / (h * h)
    n = cfg.shape[1]
    idx = np.arange(n)
    A[:, idx, idx] += lam[:, None] + dpr[None, :] / (cs * cs)
    rhs = -(rb + dpr[None, :] * (cfg - mid[None, :]) / cs)
    fx = np.asarray(fixed, bool)
    A[:, fx, :] = 0.0
    A[:, :, fx] = 0.0
    A[:, fx, fx] = 1.0
    rhs[:, fx] = 0.0
    delta = olm.chol_solve(A, rhs) / cs
    pn, on = _ee_norms(r, n_ee)
    mp, mo = pn.max(axis=1), on.max(axis=1)
    R = np.where((mp > 1e-2) | (mo > 0.6), 0.38,
                 np.where((mp > 1e-3) | (mo > 0.25), 0.22, np.where((mp > 2e-4) | (mo > 0.08), 0.12, 0.05)))
    dn = np.linalg.norm(delta, axis=1)
    sc = np.where(dn > R, R / (dn + 1e-18), 1.0)
    return delta * sc[:, None]


def lm_refine(seeds, noise, target_T, model, target_jnts, anc, lower, upper, fixed, *, max_iter, stall_patience,
              lambda_init, limit_prior_weight, kick_scale, eps_pos, eps_ori, coll=None):
    """-> (best_cfg [S, n], best_err [S], stop)."""
    cfg = np.array(seeds, np.float64)
    S, n = cfg.shape
    n_ee = len(target_jnts)
    lower, upper = np.asarray(lower, np.float64), np.asarray(upper, np.float64)
    fx = np.asarray(fixed, bool)

    def err_of(c):
        Tj = olm._fk(c, model)
        r, _ = olm.residual_and_jacobian(Tj, target_jnts, target_T, model, anc, want_jac=False)
        return np.sum(r * r, axis=1) + _penalty(Tj, coll)

    best_cfg = cfg.copy()
    best_err = err_of(cfg)
    lam = np.full(S, float(lambda_init))
    stall = np.zeros(S, np.int64)
    done = np.zeros(S, bool)
    stop = False
    for it in range(max_iter):
        if stop:
            done[:] = True
        if done.all():
            break
        Tj = olm._fk(cfg, model)
        r, J = olm.residual_and_jacobian(Tj, target_jnts, target_T, model, anc)
        curr = np.sum(r * r, axis=1) + _penalty(Tj, coll)
        pn, on = _ee_norms(r, n_ee)
        conv = np.all((pn < eps_pos) & (on < eps_ori), axis=1)
        if np.any(~done & conv):
            stop = True
        done |= conv
        act = ~done
        if not act.any():
            continue
        delta = _direction(r, J, cfg, lam, lower, upper, fx, limit_prior_weight, n_ee)
        best_a = np.full(S, 1e30)
        best_ai = np.zeros(S, np.int64)
        searching = act.copy()
        for ai, al in enumerate(ALPHAS):
            if not searching.any():
                break
            trial = np.clip(cfg + al * delta, lower, upper)
            et = err_of(trial)
            better = searching & (et < best_a)
            best_a = np.where(better, et, best_a)
            best_ai = np.where(better, ai, best_ai)
            searching &= ~(better & (et < curr * (1.0 - 1e-4)))
        alpha = np.asarray(ALPHAS)[best_ai]
        trial = np.clip(cfg + alpha[:, None] * delta, lower, upper)
        improved = act & (best_a < curr * (1.0 - 1e-4))
        rejected = act & ~improved
        cfg = np.where(improved[:, None], trial, cfg)
        lam = np.where(improved, np.maximum(lam * 0.5, 1e-10), np.where(rejected, np.minimum(lam * 3.0, 1e6), lam))
        stall = np.where(improved, 0, np.where(rejected, stall + 1, stall))
        nb = act & (best_a < best_err)
        best_err = np.where(nb, best_a, best_err)
        best_cfg = np.where(nb[:, None], trial, best_cfg)
        kick = act & (stall >= stall_patience)
        if kick.any():
            kicked = np.where(fx[None, :], cfg, np.clip(cfg + noise[:, it, :] * kick_scale, lower, upper))
            cfg = np.where(kick[:, None], kicked, cfg)
            lam = np.where(kick, float(lambda_init), lam)
            stall = np.where(kick, 0, stall)
    return best_cfg, best_err, stop
