"""GPU SCO (``pyroffi_b200.sco``) against the FP64 oracle (``oracle/sco.py``):
group distances, analytic and central-difference Jacobians, the ranking
collision sum, the inner L-BFGS solve, the ranking cost, the whole loop; the
single-call loop against the staged calls and its CUDA-graph replay."""

import numpy as np
import pytest
import torch

from oracle import sco as osco
from pyroffi_b200 import workloads as W
from pyroffi_b200.sco import ScoConfig, ScoOptimizer

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
TAU = 0.05


def scene(Bt=3, T=12, seed=1006):
    return W.mixed_trajectories(Bt=Bt, T=T, seed=seed)


def oracle_args(w):
    return (w.model.as_dict(), w.spheres.centers, w.spheres.radii, w.link_pairs, w.world.arrays())


def make(w, cfg=ScoConfig(), **kw):
    return ScoOptimizer(w.model, w.spheres, w.world, w.link_pairs, cfg, device=DEV, **kw)


@pytest.mark.parametrize("self_all", [True, False])
def test_group_distances_and_coll_sum(self_all):
    w = scene()
    opt = make(w, self_all_pairs=self_all)
    q = w.traj.reshape(-1, w.traj.shape[-1])
    d, _, c = opt.linearize(torch.as_tensor(q, device=DEV), want_jac=False, want_coll=True)
    od = osco.group_dists(q, *oracle_args(w), TAU, self_all)
    np.testing.assert_allclose(d.cpu().numpy(), od, atol=1e-5, rtol=1e-6)
    oc = osco.coll_sum(q, *oracle_args(w), 0.01, self_all)
    np.testing.assert_allclose(c.cpu().numpy(), oc, rtol=1e-5, atol=1e-6)


def test_empty_groups_read_1e10_with_zero_jacobian():
    w = scene(Bt=1, T=6)
    w.world.capsules = np.zeros((0, 7), np.float32)
    w.world.halfspaces = np.zeros((0, 6), np.float32)
    opt = make(w)
    d, J, _ = opt.linearize(torch.as_tensor(w.traj[0], device=DEV))
    d, J = d.cpu().numpy(), J.cpu().numpy()
    assert np.all(d[:, 2] == 1e10) and np.all(d[:, 4] == 1e10)
    assert np.all(J[:, 2] == 0) and np.all(J[:, 4] == 0)
    assert np.all(d[:, [0, 1, 3]] < 1e9)


@pytest.mark.parametrize("self_all", [True, False])
def test_analytic_jacobian_matches_fp64_differences(self_all):
    w = scene()
    opt = make(w, self_all_pairs=self_all)
    q = w.traj.reshape(-1, w.traj.shape[-1])
    _, J, _ = opt.linearize(torch.as_tensor(q, device=DEV))
    oJ = osco.group_jacobian(q, *oracle_args(w), TAU, self_all, eps=1e-6)
    np.testing.assert_allclose(J.cpu().numpy(), oJ, atol=2e-4, rtol=1e-3)


def test_fd_jacobian_as_the_reference_kernel():
    # central differences with the reference kernel's float32 step 1e-4
    w = scene()
    opt = make(w)
    q = torch.as_tensor(w.traj.reshape(-1, w.traj.shape[-1]), device=DEV)
    d_fd, J_fd = opt.linearize_fd(q, 1e-4)
    d, J, _ = opt.linearize(q)
    np.testing.assert_allclose(d_fd.cpu().numpy(), d.cpu().numpy(), rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(J_fd.cpu().numpy(), J.cpu().numpy(), atol=3e-3, rtol=2e-2)


def test_inner_solve_matches_oracle():
    w = scene()
    cfg = ScoConfig()
    opt = make(w, cfg)
    B, T, n = w.traj.shape
    q = w.traj.copy()
    q[:, 0], q[:, -1] = q[0, 0], q[0, -1]
    dk = np.stack([osco.group_dists(q[b], *oracle_args(w), TAU) for b in range(B)])
    Jk = np.stack([osco.group_jacobian(q[b], *oracle_args(w), TAU) for b in range(B)])
    dk32, Jk32 = dk.astype(np.float32), Jk.astype(np.float32)
    for w_coll in (1.0, 27.0):
        got = opt.inner(torch.as_tensor(q, device=DEV), torch.as_tensor(dk32, device=DEV),
                        torch.as_tensor(Jk32, device=DEV), w_coll, torch.as_tensor(q[0, 0], device=DEV),
                        torch.as_tensor(q[0, -1], device=DEV)).cpu().numpy()
        lo, hi = w.model.lower.astype(np.float64), w.model.upper.astype(np.float64)
        for b in range(B):
            ox = osco.lbfgs_inner(q[b].astype(np.float64), dk32[b].astype(np.float64), Jk32[b].astype(np.float64),
                                  lo, hi, cfg, w_coll)
            args = (q[b].astype(np.float64), dk32[b].astype(np.float64), Jk32[b].astype(np.float64), lo, hi, cfg,
                    w_coll)
            c_gpu, c_or, c0 = osco.model_cost(got[b], *args), osco.model_cost(ox, *args), osco.model_cost(q[b], *args)
            assert c_gpu <= c0
            assert abs(c_gpu - c_or) <= 1e-4 * abs(c0 - c_or) + 1e-6 * abs(c_or)
            np.testing.assert_allclose(got[b], ox, atol=2e-3)
            np.testing.assert_array_equal(got[b, 0], q[0, 0])
            np.testing.assert_array_equal(got[b, -1], q[0, -1])


def test_final_cost_matches_oracle():
    w = scene()
    cfg = ScoConfig()
    opt = make(w, cfg)
    c = opt.final_cost(torch.as_tensor(w.traj, device=DEV)).cpu().numpy()
    for b in range(w.traj.shape[0]):
        oc = osco.ranking_cost(w.traj[b], *oracle_args(w), w.model.lower, w.model.upper, cfg)
        np.testing.assert_allclose(c[b], oc, rtol=2e-5)


@pytest.mark.parametrize("fd_eps", [0.0, 1e-4])
def test_single_call_equals_staged_calls(fd_eps):
    w = scene()
    cfg = ScoConfig(n_outer_iters=3, n_inner_iters=12)
    opt = make(w, cfg, fd_eps=fd_eps)
    x = torch.as_tensor(w.traj, device=DEV)
    st, gl = x[0, 0].clone(), x[0, -1].clone()
    _, c1, f1 = opt.run(x, st, gl)
    _, c2, f2 = opt.run_stages(x, st, gl)
    np.testing.assert_array_equal(f1.cpu().numpy(), f2.cpu().numpy())
    np.testing.assert_array_equal(c1.cpu().numpy(), c2.cpu().numpy())


def test_whole_loop_against_oracle():
    w = scene()
    cfg = ScoConfig(n_outer_iters=3, n_inner_iters=15)
    opt = make(w, cfg)
    x = torch.as_tensor(w.traj, device=DEV)
    start, goal = w.traj[0, 0], w.traj[0, -1]
    best, costs, final = opt.run(x, torch.as_tensor(start, device=DEV), torch.as_tensor(goal, device=DEV))
    final, costs = final.cpu().numpy(), costs.cpu().numpy()
    lo, hi = w.model.lower, w.model.upper
    for b in range(w.traj.shape[0]):
        ox, oc = osco.sco_single(w.traj[b], start, goal, *oracle_args(w), lo, hi, cfg)
        c0 = osco.ranking_cost(w.traj[b], *oracle_args(w), lo, hi, cfg)
        assert costs[b] < c0
        np.testing.assert_allclose(costs[b], oc, rtol=2e-2)
        np.testing.assert_allclose(final[b], ox, atol=2e-2)
        np.testing.assert_array_equal(final[b, 0], start)
        np.testing.assert_array_equal(final[b, -1], goal)
    np.testing.assert_array_equal(best.cpu().numpy(), final[int(np.argmin(costs))])


def test_graph_replay_equals_eager():
    w = scene(Bt=4, T=16)
    cfg = ScoConfig(n_outer_iters=2, n_inner_iters=10)
    opt = make(w, cfg)
    x = torch.as_tensor(w.traj, device=DEV)
    st, gl = x[0, 0].clone(), x[0, -1].clone()
    _, c1, f1 = opt.run(x, st, gl)
    c1, f1 = c1.clone(), f1.clone()
    for _ in range(2):
        _, c2, f2 = opt.run(x, st, gl, graph=True)
        np.testing.assert_array_equal(f1.cpu().numpy(), f2.cpu().numpy())
        np.testing.assert_array_equal(c1.cpu().numpy(), c2.cpu().numpy())


def test_history_in_global_memory_matches_oracle():
    # a long trajectory whose L-BFGS history does not fit in shared memory
    # takes the global-history kernel; it must agree with the oracle as well
    w = W.mixed_trajectories(Bt=2, T=400, seed=7)
    cfg = ScoConfig(n_inner_iters=6, m_lbfgs=8)
    opt = make(w, cfg)
    q = w.traj.copy()
    q[:, 0], q[:, -1] = q[0, 0], q[0, -1]
    d, J, _ = opt.linearize(torch.as_tensor(q, device=DEV))
    got = opt.inner(torch.as_tensor(q, device=DEV), d, J, 3.0, torch.as_tensor(q[0, 0], device=DEV),
                    torch.as_tensor(q[0, -1], device=DEV)).cpu().numpy()
    dk, Jk = d.cpu().numpy().astype(np.float64), J.cpu().numpy().astype(np.float64)
    lo, hi = w.model.lower.astype(np.float64), w.model.upper.astype(np.float64)
    for b in range(2):
        ox = osco.lbfgs_inner(q[b].astype(np.float64), dk[b], Jk[b], lo, hi, cfg, 3.0)
        np.testing.assert_allclose(got[b], ox, atol=2e-3)


def test_invalid_arguments_raise():
    w = scene(Bt=1, T=6)
    with pytest.raises(ValueError):
        ScoOptimizer(w.model, w.spheres, w.world, np.array([[2, 2]]), device=DEV)
    from pyroffi_b200._lib import PkError
    opt = make(w, ScoConfig(m_lbfgs=0))
    with pytest.raises(PkError):
        opt.linearize(torch.as_tensor(w.traj[0], device=DEV))


@pytest.mark.parametrize("per_link", [8, 16, 20])
def test_sphere_count_variants_match_oracle(per_link):
    """The linearisation is compiled for up to 4, 8, 16 and 32 spheres per link
    (register pairs); the mixed scene at 8, 16 and 20 spheres per link takes
    the last three."""
    w = W.mixed_trajectories(Bt=2, T=8, per_link=per_link)
    opt = make(w)
    q = w.traj.reshape(-1, w.traj.shape[-1])
    d, J, c = opt.linearize(torch.as_tensor(q, device=DEV), want_coll=True)
    np.testing.assert_allclose(d.cpu().numpy(), osco.group_dists(q, *oracle_args(w), TAU, True), atol=1e-5, rtol=1e-6)
    np.testing.assert_allclose(c.cpu().numpy(), osco.coll_sum(q, *oracle_args(w), 0.01, True), rtol=1e-5, atol=1e-6)
    oJ = osco.group_jacobian(q, *oracle_args(w), TAU, True, eps=1e-6)
    np.testing.assert_allclose(J.cpu().numpy(), oJ, atol=2e-4, rtol=1e-3)
