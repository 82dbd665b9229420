"""Host-side model logic (topological order, depth schedule, ancestor masks,
sphere flattening, self pairs) against the oracle's restatement."""

import numpy as np
import pytest

from oracle import kinematics as okin
from pyroffi_b200 import robot as R
from pyroffi_b200 import workloads as W


def robots():
    rng = np.random.default_rng(5)
    return [R.serial_chain(7, rng), R.serial_chain(6, rng), R.bimanual_tree(rng), R.humanoid_tree(rng)]


@pytest.mark.parametrize("model", robots(), ids=lambda m: m.name)
def test_topo_and_schedule_match_oracle(model):
    np.testing.assert_array_equal(model.topo_inv, okin.topo_sort(model.parent_idx))
    s, j, L = okin.fk_depth_schedule(model.parent_idx, model.topo_inv)
    np.testing.assert_array_equal(model.fk_level_starts, s)
    np.testing.assert_array_equal(model.fk_level_joints, j)
    assert model.n_levels == L


def test_out_of_order_topology():
    parent = np.array([2, -1, 1, 0, 2, 3])
    np.testing.assert_array_equal(R.topo_sort(parent), okin.topo_sort(parent))
    with pytest.raises(ValueError):
        R.topo_sort([1, 0])


@pytest.mark.parametrize("model", robots(), ids=lambda m: m.name)
def test_ancestor_mask(model):
    for link in range(model.n_links):
        j = model.link_joint(link)
        expect = okin.ancestor_mask(j, model.parent_idx) if j >= 0 else np.zeros(model.n_joints, np.int32)
        np.testing.assert_array_equal(model.ancestor_mask(link), expect)


def test_robot_shapes():
    rng = np.random.default_rng(0)
    bi = R.bimanual_tree(rng)
    assert (bi.n_joints, bi.n_act, bi.n_links) == (16, 15, 17)
    hu = R.humanoid_tree(rng)
    assert (hu.n_joints, hu.n_act, hu.n_links) == (29, 29, 30)
    c = R.serial_chain(7, rng)
    assert (c.n_joints, c.n_act, c.n_links, c.n_levels) == (7, 7, 8, 7)


def test_ik_workload_is_deterministic_and_consistent():
    a, b = W.ik(P=8, Sd=4), W.ik(P=8, Sd=4)
    np.testing.assert_array_equal(a.seeds, b.seeds)
    np.testing.assert_array_equal(a.self_pairs, b.self_pairs)
    assert a.spheres_local.shape == (56, 4) and a.sphere_joint.shape == (56,)
    assert a.self_pairs.shape == (200, 2)
    assert np.all(a.seeds >= a.model.lower) and np.all(a.seeds <= a.model.upper)
    # sphere k of the flat list sits on link (joint + 1); pairs are non-adjacent
    link = a.sphere_joint + 1
    li, lj = link[a.self_pairs[:, 0]], link[a.self_pairs[:, 1]]
    assert np.all(np.abs(li - lj) >= 2)
    assert len({tuple(p) for p in a.self_pairs}) == 200


def test_fk_collision_workload():
    w = W.fk_collision(B=16)
    assert w.cfg.shape == (16, 7) and w.world.spheres.shape == (64, 4)
    assert w.spheres.centers.shape == (8, 8, 3)
    assert np.all(w.spheres.radii[0] < 0)                # base link: padding only
    assert np.all((w.spheres.radii[1:] >= 0.03) & (w.spheres.radii[1:] <= 0.08))


def test_trajectory_workload():
    w = W.trajectories(Bt=4, T=16)
    assert w.traj.shape == (4, 16, 7)
    assert w.world.spheres.shape == (256, 4) and w.world.boxes.shape == (32, 15)
    np.testing.assert_allclose(w.world.boxes[:, 3:12], np.tile(np.eye(3).T.reshape(-1), (32, 1)))
    # active pairs: 8-link chain, links with spheres 1..7, minus 6 adjacent pairs
    assert w.link_pairs.shape == (15, 2)
