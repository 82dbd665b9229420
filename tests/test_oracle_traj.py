"""The trajectory-cost oracle: analytic smoothness / limit gradients against
central differences, and the collision cost's structure."""

import numpy as np

from oracle import traj as otr
from pyroffi_b200 import workloads as W


def test_smoothness_gradient_matches_fd():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(12, 3))
    g = otr.smoothness_grad(x, 0.5, 0.1)
    h = 1e-6
    fd = np.zeros_like(x)
    for i in np.ndindex(x.shape):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd[i] = (otr.smoothness(xp, 0.5, 0.1) - otr.smoothness(xm, 0.5, 0.1)) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-6)


def test_smoothness_of_linear_motion_is_zero():
    x = np.linspace(0, 1, 20)[:, None] * np.array([[1.0, -2.0]])
    assert otr.smoothness(x, 0.5, 0.1) < 1e-20


def test_limits_gradient():
    x = np.array([[0.5, 3.0], [-4.0, 0.0]])
    lo, hi = np.array([-2.8, -2.8]), np.array([2.8, 2.8])
    assert np.isclose(otr.limits(x, lo, hi), 0.2 ** 2 + 1.2 ** 2)
    np.testing.assert_allclose(otr.limits_grad(x, lo, hi), [[0, 0.4], [-2.4, 0]])


def test_collision_cost_nonnegative_and_zero_without_world():
    w = W.trajectories(Bt=2, T=8)
    md = w.model.as_dict()
    empty = [np.zeros((0, k)) for k in (4, 7, 15, 6)]
    c0 = otr.collision_cost(w.traj[0], md, w.spheres.centers, w.spheres.radii, np.zeros((0, 2), int), empty,
                            w.margin)
    assert c0 == 0.0
    c1 = otr.collision_cost(w.traj[0], md, w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays(),
                            w.margin)
    assert c1 >= 0.0
