"""GPU parity of the trajectory cost and its hand-written adjoint: cost
against the FP64 oracle, gradient against the oracle's analytic smoothness /
limit gradient plus FP64 central differences of the collision cost
(relative error <= 1e-4), and the torch.autograd adapter."""

import numpy as np
import pytest
import torch

from error_report import record
from oracle import traj as otr
from pyroffi_b200 import workloads as W
from pyroffi_b200.trajopt import TrajectoryCost, TrajectoryCostFn

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def setup(Bt=4, T=16, seed=1003):
    w = W.trajectories(Bt=Bt, T=T, seed=seed)
    tc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=w.margin, w_smooth=w.w_smooth,
                        w_acc=w.w_acc, w_jerk=w.w_jerk, w_limits=w.w_limits, w_coll=w.w_collision, device=DEV)
    return w, tc


def oracle_cost(w, x):
    return otr.total_cost(x, w.model.as_dict(), w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays(),
                          margin=w.margin, w_smooth=w.w_smooth, w_acc=w.w_acc, w_jerk=w.w_jerk,
                          w_limits=w.w_limits, w_coll=w.w_collision, lower=w.model.lower, upper=w.model.upper)


def test_cost_matches_oracle():
    w, tc = setup(Bt=16, T=32)
    c = tc.cost(torch.as_tensor(w.traj, device=DEV)).cpu().numpy()
    ref = np.array([oracle_cost(w, w.traj[b].astype(np.float64)) for b in range(16)])
    record("trajectory cost (relative)", np.abs(c - ref) / np.abs(ref), "16 x 32 x 7")
    np.testing.assert_allclose(c, ref, rtol=1e-4, atol=1e-5)
    wp = tc.waypoint_collision(torch.as_tensor(w.traj, device=DEV)).cpu().numpy()
    assert (wp > 0).any(), "the workload should touch obstacles"


def test_gradient_matches_finite_differences():
    w, tc = setup(Bt=3, T=12)
    x = torch.as_tensor(w.traj, device=DEV)
    c, g = tc.cost_and_grad(x)
    g = g.cpu().numpy().astype(np.float64)
    md = w.model.as_dict()
    for b in range(3):
        xb = w.traj[b].astype(np.float64)
        ref = (w.w_smooth * otr.smoothness_grad(xb, w.w_acc, w.w_jerk)
               + w.w_limits * otr.limits_grad(xb, w.model.lower, w.model.upper)
               + w.w_collision * otr.collision_grad_fd(xb, md, w.spheres.centers, w.spheres.radii, w.link_pairs,
                                                       w.world.arrays(), w.margin))
        rel = np.linalg.norm(g[b] - ref) / max(np.linalg.norm(ref), 1e-12)
        record("trajectory gradient vs FP64 finite differences (relative)", rel, "3 x 12 x 7, full cost")
        assert rel < 1e-4, (b, rel)
    # the fused launch and the separate ones agree
    np.testing.assert_allclose(tc.cost(x).cpu().numpy(), c.cpu().numpy(), rtol=0, atol=0)
    np.testing.assert_allclose(tc.grad(x).cpu().numpy(), g.astype(np.float32), rtol=0, atol=0)


def test_collision_gradient_alone_matches_fd():
    """Collision-only weights, waypoints that touch obstacles."""
    w, _ = setup(Bt=8, T=8)
    tc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=w.margin, w_smooth=0.0, w_acc=0.0,
                        w_jerk=0.0, w_limits=0.0, w_coll=1.0, device=DEV)
    x = torch.as_tensor(w.traj, device=DEV)
    wp = tc.waypoint_collision(x).cpu().numpy()
    b = int(np.argmax(wp.sum(1)))
    assert wp[b].sum() > 0
    g = tc.grad(x).cpu().numpy()[b].astype(np.float64)
    ref = otr.collision_grad_fd(w.traj[b].astype(np.float64), w.model.as_dict(), w.spheres.centers,
                                w.spheres.radii, w.link_pairs, w.world.arrays(), w.margin)
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    record("trajectory gradient vs FP64 finite differences (relative)", rel, "8 x 8 x 7, collision only")
    assert rel < 1e-4, rel


def test_autograd_adapter():
    w, tc = setup(Bt=4, T=16)
    x = torch.as_tensor(w.traj, device=DEV).requires_grad_(True)
    J = TrajectoryCostFn.apply(x, tc)
    (J * torch.arange(1, 5, device=DEV, dtype=J.dtype)).sum().backward()
    _, g = tc.cost_and_grad(x.detach())
    np.testing.assert_allclose(x.grad.cpu().numpy(), (g * torch.arange(1, 5, device=DEV)[:, None, None]).cpu().numpy(),
                               rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("margin,n_spheres", [(0.01, 24), (0.3, 23)])
def test_all_obstacle_kinds_match_oracle(margin, n_spheres):
    """Spheres, capsules, oriented boxes and a halfspace (each kind has its own
    broad-phase loop; the spheres go two per packed test, so an odd count pads
    the last pair); the large margin keeps most (link, obstacle) pairs and puts
    link bounding centres inside boxes."""
    w = W.mixed_trajectories(Bt=6, T=12, n_spheres=n_spheres)
    tc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=margin, w_smooth=1.0, w_acc=0.5,
                        w_jerk=0.1, w_limits=1.0, w_coll=3.0, device=DEV)
    x = torch.as_tensor(w.traj, device=DEV)
    c, g = tc.cost_and_grad(x)
    md = w.model.as_dict()
    for b in range(6):
        xb = w.traj[b].astype(np.float64)
        ref = otr.total_cost(xb, md, w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays(),
                             margin=margin, w_smooth=1.0, w_acc=0.5, w_jerk=0.1, w_limits=1.0, w_coll=3.0,
                             lower=w.model.lower, upper=w.model.upper)
        assert abs(float(c[b]) - ref) <= 1e-4 * abs(ref) + 1e-5, (b, float(c[b]), ref)
    b = int(np.argmax(tc.waypoint_collision(x).cpu().numpy().sum(1)))
    tcc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=margin, w_smooth=0.0, w_acc=0.0,
                         w_jerk=0.0, w_limits=0.0, w_coll=1.0, device=DEV)
    gc = tcc.grad(x).cpu().numpy()[b].astype(np.float64)
    ref = otr.collision_grad_fd(w.traj[b].astype(np.float64), md, w.spheres.centers, w.spheres.radii, w.link_pairs,
                                w.world.arrays(), margin)
    assert np.linalg.norm(ref) > 0
    assert np.linalg.norm(gc - ref) / np.linalg.norm(ref) < 1e-4


def test_large_batch_two_lane_path_matches_oracle():
    """Batches above 2 x SMs run 2 lanes per waypoint (config 3 and the CHOMP
    line search take that path); smaller ones 4.  Both against the oracle, and
    against each other on the same trajectories."""
    w, tc = setup(Bt=320, T=16)
    x = torch.as_tensor(w.traj, device=DEV)
    c_big, g_big = tc.cost_and_grad(x)
    c_small, g_small = tc.cost_and_grad(x[:12].contiguous())
    np.testing.assert_allclose(c_big[:12].cpu().numpy(), c_small.cpu().numpy(), rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(g_big[:12].cpu().numpy(), g_small.cpu().numpy(), rtol=1e-4, atol=1e-5)
    idx = [0, 5, 77, 150, 233, 319]
    ref = np.array([oracle_cost(w, w.traj[b].astype(np.float64)) for b in idx])
    np.testing.assert_allclose(c_big.cpu().numpy()[idx], ref, rtol=1e-4, atol=1e-5)
    md = w.model.as_dict()
    for b in (77, 319):
        xb = w.traj[b].astype(np.float64)
        ref_g = (w.w_smooth * otr.smoothness_grad(xb, w.w_acc, w.w_jerk)
                 + w.w_limits * otr.limits_grad(xb, w.model.lower, w.model.upper)
                 + w.w_collision * otr.collision_grad_fd(xb, md, w.spheres.centers, w.spheres.radii, w.link_pairs,
                                                         w.world.arrays(), w.margin))
        rel = np.linalg.norm(g_big[b].cpu().numpy() - ref_g) / max(np.linalg.norm(ref_g), 1e-12)
        assert rel < 1e-4, (b, rel)


@pytest.mark.parametrize("per_link", [8, 16, 20])
def test_sphere_count_variants_match_oracle(per_link):
    """Kernels for up to 8, 16 and 32 spheres per link (register pairs)."""
    w = W.mixed_trajectories(Bt=3, T=10, per_link=per_link)
    margin = 0.05
    tc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=margin, w_smooth=1.0, w_acc=0.5,
                        w_jerk=0.1, w_limits=1.0, w_coll=3.0, device=DEV)
    x = torch.as_tensor(w.traj, device=DEV)
    c = tc.cost(x).cpu().numpy()
    md = w.model.as_dict()
    for b in range(3):
        ref = otr.total_cost(w.traj[b].astype(np.float64), md, w.spheres.centers, w.spheres.radii, w.link_pairs,
                             w.world.arrays(), margin=margin, w_smooth=1.0, w_acc=0.5, w_jerk=0.1, w_limits=1.0,
                             w_coll=3.0, lower=w.model.lower, upper=w.model.upper)
        assert abs(float(c[b]) - ref) <= 1e-4 * abs(ref) + 1e-5, (b, float(c[b]), ref)
    tcc = TrajectoryCost(w.model, w.spheres, w.world, w.link_pairs, margin=margin, w_smooth=0.0, w_acc=0.0,
                         w_jerk=0.0, w_limits=0.0, w_coll=1.0, device=DEV)
    b = int(np.argmax(tcc.waypoint_collision(x).cpu().numpy().sum(1)))
    g = tcc.grad(x).cpu().numpy()[b].astype(np.float64)
    ref = otr.collision_grad_fd(w.traj[b].astype(np.float64), md, w.spheres.centers, w.spheres.radii, w.link_pairs,
                                w.world.arrays(), margin)
    assert np.linalg.norm(ref) > 0
    assert np.linalg.norm(g - ref) / np.linalg.norm(ref) < 1e-4
