"""SCO oracle (``oracle/sco.py``) self-checks on the CPU: smooth minimum
bounds, the convex model's gradient against central differences, the inner
L-BFGS against the model's exact minimiser, the group distances against a
brute-force restatement, and the host-side pieces of ``pyroffi_b200.sco``."""

import numpy as np
import pytest

from oracle import collision as ocoll
from oracle import sco as osco
from pyroffi_b200 import workloads as W
from pyroffi_b200.sco import ScoConfig, make_init_trajs


def test_smooth_min_bounds():
    rng = np.random.default_rng(0)
    for k in (1, 5, 200):
        d = rng.uniform(-0.1, 1.0, k)
        s = osco.smooth_min(d, 0.05)
        assert s <= d.min() + 1e-12
        assert s >= d.min() - 0.05 * np.log(k) - 1e-12
    assert osco.smooth_min(np.zeros(0), 0.05) == 1e10
    assert abs(osco.smooth_min(np.array([0.3]), 0.05) - 0.3) < 1e-15


def _model_problem(seed=0, T=16, n=3):
    rng = np.random.default_rng(seed)
    qk = np.cumsum(rng.normal(0, 0.1, (T, n)), axis=0)
    dk = rng.uniform(-0.05, 0.1, (T, 5))
    Jk = rng.normal(0, 0.5, (T, 5, n))
    lower, upper = -np.ones(n), np.ones(n)
    return qk, dk, Jk, lower, upper


def test_model_gradient_matches_central_differences():
    qk, dk, Jk, lo, hi = _model_problem()
    cfg = ScoConfig()
    x = qk + np.random.default_rng(1).normal(0, 0.05, qk.shape)
    g = osco.model_grad(x, qk, dk, Jk, lo, hi, cfg, 7.0)
    h = 1e-6
    for t in range(1, x.shape[0] - 1):
        for d in range(x.shape[1]):
            xp, xm = x.copy(), x.copy()
            xp[t, d] += h
            xm[t, d] -= h
            fd = (osco.model_cost(xp, qk, dk, Jk, lo, hi, cfg, 7.0) - osco.model_cost(xm, qk, dk, Jk, lo, hi, cfg,
                                                                                       7.0)) / (2 * h)
            assert abs(fd - g[t, d]) < 1e-6 * (1 + abs(fd))
    assert np.all(g[0] == 0) and np.all(g[-1] == 0)


def test_inner_lbfgs_approaches_the_quadratic_minimiser():
    # without active collision or limit terms the model is quadratic:
    # (w_smooth H + w_trust I) on the interior, endpoints fixed
    qk, _, _, lo, hi = _model_problem(2, T=24, n=2)
    qk *= 0.2
    dk = np.full((qk.shape[0], 5), 1.0)          # far from the margin: hinge inactive
    Jk = np.zeros((qk.shape[0], 5, qk.shape[1]))
    cfg = ScoConfig(n_inner_iters=60)
    x = osco.lbfgs_inner(qk, dk, Jk, lo, hi, cfg, 1.0)
    T, n = qk.shape
    # exact minimiser: stack the interior coordinates and solve the normal equations
    idx = [(t, d) for t in range(1, T - 1) for d in range(n)]
    A = np.zeros((len(idx), len(idx)))
    b = np.zeros(len(idx))
    f0 = lambda z: osco.model_cost(z, qk, dk, Jk, lo, hi, cfg, 1.0)  # noqa: E731
    base = qk.copy()
    g0 = osco.model_grad(base, qk, dk, Jk, lo, hi, cfg, 1.0)
    for k, (t, d) in enumerate(idx):
        e = np.zeros_like(qk)
        e[t, d] = 1.0
        col = osco.model_grad(base + e, qk, dk, Jk, lo, hi, cfg, 1.0) - g0
        A[:, k] = [col[tt, dd] for tt, dd in idx]
        b[k] = -g0[t, d]
    step = np.linalg.solve(A, b)
    xopt = base.copy()
    for k, (t, d) in enumerate(idx):
        xopt[t, d] += step[k]
    c0, c, copt = f0(qk), f0(x), f0(xopt)
    assert c <= c0
    assert c - copt <= 1e-4 * (c0 - copt)
    np.testing.assert_array_equal(x[0], qk[0])
    np.testing.assert_array_equal(x[-1], qk[-1])


def test_group_distances_match_brute_force():
    w = W.mixed_trajectories(Bt=1, T=6)
    m = w.model.as_dict()
    cen, rad = osco.link_spheres_world(w.traj[0], m, w.spheres.centers, w.spheres.radii)
    pd = osco.pair_distances(w.traj[0], m, w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays())
    ws, wc, wb, wh = (np.asarray(a, np.float64) for a in w.world.arrays())
    for c in range(w.traj.shape[1]):
        # self: every sphere pair of every active pair
        want = []
        for li, lj in w.link_pairs:
            best = np.inf
            for a in range(rad.shape[1]):
                for b in range(rad.shape[1]):
                    if rad[li, a] < 0 or rad[lj, b] < 0:
                        continue
                    best = min(best, np.linalg.norm(cen[c, li, a] - cen[c, lj, b]) - rad[li, a] - rad[lj, b])
            if np.isfinite(best):
                want.append(best)
        np.testing.assert_allclose(pd[c][0], want, rtol=0, atol=1e-12)
        # world spheres: per (link, obstacle) minimum over the link's spheres
        got = pd[c][1].reshape(-1, len(ws))
        k = 0
        for l in range(rad.shape[0]):
            v = rad[l] >= 0
            if not v.any():
                continue
            d = ocoll.sphere_sphere(cen[c, l][v][:, None], rad[l][v][:, None], ws[:, :3], ws[:, 3]).min(0)
            np.testing.assert_allclose(got[k], d, atol=1e-12)
            k += 1
    g = osco.group_dists(w.traj[0], m, w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays(), 0.05)
    for c in range(w.traj.shape[1]):
        for k in range(5):
            assert g[c, k] <= pd[c][k].min() + 1e-12


def test_equal_index_self_distance_is_an_upper_bound():
    w = W.mixed_trajectories(Bt=1, T=4)
    m = w.model.as_dict()
    a = osco.pair_distances(w.traj[0], m, w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays(), True)
    b = osco.pair_distances(w.traj[0], m, w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays(), False)
    for c in range(len(a)):
        assert np.all(b[c][0] >= a[c][0] - 1e-12)


def test_make_init_trajs_shape_and_ends():
    s, g = np.zeros(3), np.ones(3)
    x = make_init_trajs(s, g, 5, 9, noise_scale=0.0)
    assert x.shape == (5, 9, 3) and x.dtype == np.float32
    np.testing.assert_allclose(x[:, 0], 0.0)
    np.testing.assert_allclose(x[:, -1], 1.0)


@pytest.mark.parametrize("self_all", [True, False])
def test_sco_single_lowers_the_ranking_cost(self_all):
    w = W.mixed_trajectories(Bt=1, T=10)
    m = w.model.as_dict()
    cfg = ScoConfig(n_outer_iters=2, n_inner_iters=8)
    args = (m, w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays())
    x, c = osco.sco_single(w.traj[0], w.traj[0, 0], w.traj[0, -1], *args, w.model.lower, w.model.upper, cfg,
                           self_all=self_all)
    c0 = osco.ranking_cost(w.traj[0], *args, w.model.lower, w.model.upper, cfg, self_all=self_all)
    assert c < c0
    np.testing.assert_array_equal(x[0], w.traj[0, 0])
    np.testing.assert_array_equal(x[-1], w.traj[0, -1])
