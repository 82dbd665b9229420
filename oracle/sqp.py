"""SQP-IK -- FP64 oracle (test infrastructure only).

Restates ``sqp_ik_kernel`` (``src/pyroffi/cuda_kernels/_sqp_ik_cuda_kernel.cu:70-460``)
for the seeds of one problem, vectorised with numpy.  Per iteration:

- residual / stacked Jacobian (``oracle.lm.residual_and_jacobian``), and the
  exit once every EE is within (eps_pos, eps_ori) (``:245-255``);
- rows weighted by (pos_weight, ori_weight); the error is the weighted sum
  of squares plus the hinge penalty (``:258-267``);
- Jacobi column scaling, ``H = Js^T Js + lam I``, ``g = Js^T f``
  (``:270-297``);
- the step's box in scaled space, ``((lower - q) s, (upper - q) s)``, 0 for
  fixed joints (``:300-305``);
- the Newton step ``-H^-1 g`` with fixed joints masked (Cholesky, zero step on
  a non-positive pivot), clamped to the box (``:308-331``);
- ``n_inner`` active-set re-solves: joints within 1e-8 of a bound hold their
  clamped value, the others solve ``H_ff p_f = -(g + H p_bound)_f`` and are
  clamped (``:333-363``);
- unscaling, the trust-region clip (``:366-388``);
- a 5-point line search, first minimum (``:391-418``);
- accept if ``err < curr (1 - 1e-4)`` (lambda x0.5 / x3 within [1e-10, 1e6]),
  all-time best (``:421-441``).

The reference kernel's FK ignores mimic joints; the restatement uses the
general FK, equal for robots without mimics.
"""

from __future__ import annotations

import numpy as np

from . import lm as olm
from .hjcd import _penalty

ALPHAS = (1.0, 0.5, 0.25, 0.1, 0.025)


def _weights(n_ee, pos_weight, ori_weight):
    return np.tile(np.array([pos_weight] * 3 + [ori_weight] * 3, np.float64), n_ee)


def _box_step(H, g, lb, ub, fixed, n_inner):
    """Box-constrained step in scaled space (per seed, batched)."""
    S, n = g.shape
    fx = np.asarray(fixed, bool)
    A = H.copy()
    A[:, fx, :] = 0.0
    A[:, :, fx] = 0.0
    A[:, fx, fx] = 1.0
    rhs = -g.copy()
    rhs[:, fx] = 0.0
    p = np.clip(olm.chol_solve(A, rhs), lb, ub)
    for _ in range(n_inner):
        act = (p <= lb + 1e-8) | (p >= ub - 1e-8)
        pb = np.where(act, np.clip(p, lb, ub), 0.0)
        rhs = np.where(act, 0.0, -(g + np.einsum("sij,sj->si", H, pb)))
        A = np.where(act[:, :, None] | act[:, None, :], 0.0, H)
        idx = np.arange(n)
        A[:, idx, idx] = np.where(act, 1.0, A[:, idx, idx])
        x = olm.chol_solve(A, rhs)
        p = np.where(act, pb, np.clip(x, lb, ub))
    return p


def sqp(seeds, target_T, model, target_jnts, anc, lower, upper, fixed, *, max_iter, n_inner, pos_weight,
        ori_weight, lambda_init, eps_pos, eps_ori, coll=None):
    """-> (best_cfg [S, n], best_err [S])."""
    cfg = np.array(seeds, np.float64)
    S, n = cfg.shape
    n_ee = len(target_jnts)
    lower, upper = np.asarray(lower, np.float64), np.asarray(upper, np.float64)
    fx = np.asarray(fixed, bool)
    W = _weights(n_ee, pos_weight, ori_weight)

    def err_of(c):
        Tj = olm._fk(c, model)
        r, _ = olm.residual_and_jacobian(Tj, target_jnts, target_T, model, anc, want_jac=False)
        return np.sum((r * W) ** 2, axis=1) + _penalty(Tj, coll)

    best_cfg = cfg.copy()
    best_err = err_of(cfg)
    lam = np.full(S, float(lambda_init))
    done = np.zeros(S, bool)
    for _ in range(max_iter):
        Tj = olm._fk(cfg, model)
        r, J = olm.residual_and_jacobian(Tj, target_jnts, target_T, model, anc)
        rr = r.reshape(S, n_ee, 6)
        pn, on = np.linalg.norm(rr[..., :3], axis=-1), np.linalg.norm(rr[..., 3:], axis=-1)
        done |= np.all((pn < eps_pos) & (on < eps_ori), axis=1)
        act = ~done
        if not act.any():
            break
        curr = np.sum((r * W) ** 2, axis=1) + _penalty(Tj, coll)
        fw = r * W
        Jw = J * W[None, :, None]
        cs = np.sqrt(np.sum(Jw * Jw, axis=1)) + 1e-8
        Js = Jw / cs[:, None, :]
        H = np.einsum("ski,skj->sij", Js, Js)
        idx = np.arange(n)
        H[:, idx, idx] += lam[:, None]
        g = np.einsum("ski,sk->si", Js, fw)
        lb = np.where(fx[None, :], 0.0, (lower[None, :] - cfg) * cs)
        ub = np.where(fx[None, :], 0.0, (upper[None, :] - cfg) * cs)
        p = _box_step(H, g, lb, ub, fx, n_inner)
        delta = p / cs
        mp, mo = pn.max(axis=1), on.max(axis=1)
        R = np.where((mp > 1e-2) | (mo > 0.6), 0.38,
                     np.where((mp > 1e-3) | (mo > 0.25), 0.22, np.where((mp > 2e-4) | (mo > 0.08), 0.12, 0.05)))
        dn = np.linalg.norm(delta, axis=1)
        delta = delta * np.where(dn > R, R / (dn + 1e-18), 1.0)[:, None]
        trials = [np.clip(cfg + al * delta, lower, upper) for al in ALPHAS]
        errs = np.stack([err_of(t) for t in trials], axis=1)            # [S, 5]
        bi = np.argmin(errs, axis=1)
        be = errs[np.arange(S), bi]
        trial = np.stack(trials, axis=1)[np.arange(S), bi]
        improved = act & (be < curr * (1.0 - 1e-4))
        rejected = act & ~improved
        cfg = np.where(improved[:, None], trial, cfg)
        lam = np.where(improved, np.maximum(lam * 0.5, 1e-10), np.where(rejected, np.minimum(lam * 3.0, 1e6), lam))
        nb = act & (be < best_err)
        best_err = np.where(nb, be, best_err)
        best_cfg = np.where(nb[:, None], trial, best_cfg)
    return best_cfg, best_err
