"""URDF / SRDF loader (``pyroffi_b200.urdf``).

The reference's own parser needs yourdfpy, which is not installed, so the
loader is checked against the URDF rules directly: field by field on a small
robot that exercises every joint kind (revolute, continuous without limits,
prismatic, fixed with an RPY origin, a mimic, a mimic of a fixed joint,
joints listed child-before-parent), and by comparing the FP64 oracle's FK of
the parsed model with an independent 4x4 homogeneous-matrix evaluation of
the same URDF.
"""

import math

import numpy as np
import pytest
from scipy.spatial.transform import Rotation

from oracle import kinematics as okin
from pyroffi_b200.urdf import load_urdf, read_srdf_group_states, rpy_to_wxyz

URDF = """<?xml version="1.0"?>
<robot name="tester">
  <link name="base"><collision><origin xyz="0 0 0.05"/><geometry><sphere radius="0.1"/></geometry></collision></link>
  <link name="l1">
    <collision><origin xyz="0 0 0.1"/><geometry><sphere radius="0.05"/></geometry></collision>
    <collision><origin xyz="0.02 0 0.2" rpy="0.3 0 0"/><geometry><sphere radius="0.04"/></geometry></collision>
  </link>
  <link name="l2"><collision><geometry><box size="0.1 0.1 0.1"/></geometry></collision></link>
  <link name="l3">
    <collision><origin xyz="0.1 0 0"/><geometry><sphere radius="0.03"/></geometry></collision>
    <collision><origin xyz="0.2 0 0"/><geometry><sphere radius="0.03"/></geometry></collision>
    <collision><origin xyz="0.3 0 0"/><geometry><sphere radius="0.02"/></geometry></collision>
  </link>
  <link name="tool"/>
  <link name="finger_a"/>
  <link name="finger_b"/>
  <link name="cam"/>
  <joint name="j3" type="prismatic">
    <parent link="l2"/><child link="l3"/>
    <origin xyz="0 0.1 0.3" rpy="0 0.5 0"/><axis xyz="0 0 1"/>
    <limit lower="-0.1" upper="0.2" velocity="0.5" effort="10"/>
  </joint>
  <joint name="j1" type="revolute">
    <parent link="base"/><child link="l1"/>
    <origin xyz="0 0 0.2"/><axis xyz="0 0 1"/>
    <limit lower="-2" upper="2" velocity="1.5" effort="10"/>
  </joint>
  <joint name="j2" type="continuous">
    <parent link="l1"/><child link="l2"/>
    <origin xyz="0.1 0 0.25" rpy="0.2 -0.3 0.4"/><axis xyz="0 1 0"/>
    <limit velocity="2.0" effort="10"/>
  </joint>
  <joint name="tool_fixed" type="fixed">
    <parent link="l3"/><child link="tool"/>
    <origin xyz="0.35 0 0" rpy="1.5707963 0 0.7"/>
  </joint>
  <joint name="fa" type="revolute">
    <parent link="tool"/><child link="finger_a"/>
    <origin xyz="0 0.02 0"/><axis xyz="1 0 0"/>
    <limit lower="0" upper="0.8" velocity="1" effort="1"/>
  </joint>
  <joint name="fb" type="revolute">
    <parent link="tool"/><child link="finger_b"/>
    <origin xyz="0 -0.02 0"/><axis xyz="1 0 0"/>
    <limit lower="-0.8" upper="0" velocity="1" effort="1"/>
    <mimic joint="fa" multiplier="-1.0" offset="0.05"/>
  </joint>
  <joint name="cam_j" type="revolute">
    <parent link="l1"/><child link="cam"/>
    <origin xyz="0 0.05 0"/><axis xyz="0 0 1"/>
    <limit lower="-1" upper="1" velocity="1" effort="1"/>
    <mimic joint="tool_fixed" multiplier="2.0" offset="0.3"/>
  </joint>
</robot>
"""

SRDF = """<robot name="tester">
  <group_state name="home" group="arm"><joint name="j1" value="0.1"/><joint name="j2" value="-0.2"/></group_state>
  <disable_collisions link1="l1" link2="l3" reason="Never"/>
  <disable_collisions link1="base" link2="l1" reason="Adjacent"/>
</robot>
"""


def test_joint_and_link_fields():
    r = load_urdf(URDF)
    m = r.model
    assert r.joint_names == ("j3", "j1", "j2", "tool_fixed", "fa", "fb", "cam_j")
    assert r.actuated_names == ("j3", "j1", "j2", "fa")
    assert r.link_names == ("base", "l1", "l2", "l3", "tool", "finger_a", "finger_b", "cam")
    assert r.base_link == "base"
    np.testing.assert_array_equal(m.act_idx, [0, 1, 2, -1, 3, -1, -1])
    np.testing.assert_array_equal(m.mimic_act_idx, [-1, -1, -1, -1, -1, 3, -1])
    np.testing.assert_allclose(m.mimic_mul, [1, 1, 1, 1, 1, -1, 2])
    np.testing.assert_allclose(m.mimic_off, [0, 0, 0, 0, 0, 0.05, 0.3])
    np.testing.assert_array_equal(m.parent_idx, [2, -1, 1, 0, 3, 3, 1])
    np.testing.assert_array_equal(m.parent_joint_indices, [-1, 1, 2, 0, 3, 4, 5, 6])
    np.testing.assert_allclose(m.twists[0], [0, 0, 1, 0, 0, 0])
    np.testing.assert_allclose(m.twists[2], [0, 0, 0, 0, 1, 0])
    np.testing.assert_allclose(m.twists[3], 0)
    np.testing.assert_allclose(m.lower, [-0.1, -2, -math.pi, 0], rtol=1e-6)
    np.testing.assert_allclose(m.upper, [0.2, 2, math.pi, 0.8], rtol=1e-6)
    np.testing.assert_allclose(r.velocity_limits, [0.5, 1.5, 2.0, 1.0])
    # a joint is placed after its parent joint and after the joint it mimics
    pos = {int(j): k for k, j in enumerate(m.topo_inv)}
    for j in range(m.n_joints):
        if m.parent_idx[j] >= 0:
            assert pos[int(m.parent_idx[j])] < pos[j]
    assert pos[4] < pos[5]
    assert m.fk_level_starts[-1] == m.n_joints


def test_parent_transform_quaternion():
    r = load_urdf(URDF)
    q = r.model.parent_tf[2, :4].astype(np.float64)
    want = Rotation.from_euler("xyz", [0.2, -0.3, 0.4]).as_quat()  # x, y, z, w
    assert abs(abs(np.dot(q, [want[3], *want[:3]])) - 1) < 1e-6
    np.testing.assert_allclose(r.model.parent_tf[2, 4:], [0.1, 0, 0.25], atol=1e-7)
    np.testing.assert_allclose(rpy_to_wxyz(0, 0, 0), [1, 0, 0, 0])


def test_spheres_padding_and_skipped_geometry():
    r = load_urdf(URDF)
    sp = r.spheres
    assert sp.centers.shape == (8, 3, 3) and sp.radii.shape == (8, 3)
    np.testing.assert_allclose(sp.radii[0], [0.1, -1e9, -1e9])
    np.testing.assert_allclose(sp.radii[1, :2], [0.05, 0.04])
    np.testing.assert_allclose(sp.centers[1, 1], [0.02, 0, 0.2])
    assert np.all(sp.radii[2] < 0)  # box collision is not a sphere
    np.testing.assert_allclose(sp.radii[3], [0.03, 0.03, 0.02])


def test_active_pairs_adjacency_user_and_srdf():
    r = load_urdf(URDF)
    pairs = {tuple(p) for p in r.active_pairs}
    assert all(i > j for i, j in pairs)
    idx = {n: k for k, n in enumerate(r.link_names)}
    assert (idx["l1"], idx["base"]) not in pairs      # parent / child
    assert (idx["l3"], idx["l1"]) in pairs
    assert len(pairs) == 28 - 7                       # 8 links: 28 pairs, 7 joints
    r2 = load_urdf(URDF, user_ignore_pairs=[("l3", "l1")])
    assert (idx["l3"], idx["l1"]) not in {tuple(p) for p in r2.active_pairs}
    r3 = load_urdf(URDF, srdf=SRDF)
    p3 = {tuple(p) for p in r3.active_pairs}
    assert len(p3) == 28 - 2
    assert (idx["l3"], idx["l1"]) not in p3 and (idx["l2"], idx["l1"]) in p3
    assert read_srdf_group_states(SRDF) == {"arm": {"home": {"j1": 0.1, "j2": -0.2}}}


def _matrix_fk(cfg):
    """Independent 4x4 evaluation of the URDF above: link -> world transform."""
    def T(xyz, rpy):
        M = np.eye(4)
        M[:3, :3] = Rotation.from_euler("xyz", rpy).as_matrix()
        M[:3, 3] = xyz
        return M

    def rot(axis, q):
        M = np.eye(4)
        M[:3, :3] = Rotation.from_rotvec(np.asarray(axis, float) * q).as_matrix()
        return M

    def trans(axis, q):
        M = np.eye(4)
        M[:3, 3] = np.asarray(axis, float) * q
        return M

    j3, j1, j2, fa = cfg
    W = {"base": np.eye(4)}
    W["l1"] = W["base"] @ T([0, 0, 0.2], [0, 0, 0]) @ rot([0, 0, 1], j1)
    W["l2"] = W["l1"] @ T([0.1, 0, 0.25], [0.2, -0.3, 0.4]) @ rot([0, 1, 0], j2)
    W["l3"] = W["l2"] @ T([0, 0.1, 0.3], [0, 0.5, 0]) @ trans([0, 0, 1], j3)
    W["tool"] = W["l3"] @ T([0.35, 0, 0], [1.5707963, 0, 0.7])
    W["finger_a"] = W["tool"] @ T([0, 0.02, 0], [0, 0, 0]) @ rot([1, 0, 0], fa)
    W["finger_b"] = W["tool"] @ T([0, -0.02, 0], [0, 0, 0]) @ rot([1, 0, 0], -fa + 0.05)
    W["cam"] = W["l1"] @ T([0, 0.05, 0], [0, 0, 0]) @ rot([0, 0, 1], 0.3)  # mimics a fixed joint: q = offset
    return W


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_fk_of_parsed_model_matches_matrix_fk(seed):
    r = load_urdf(URDF)
    rng = np.random.default_rng(seed)
    cfg = rng.uniform(r.model.lower, r.model.upper).astype(np.float64)
    poses = okin.forward_kinematics(cfg[None], r.model.as_dict())[0]    # [N, 7] wxyz_xyz
    W = _matrix_fk(cfg)
    for n, name in enumerate(r.link_names):
        q = poses[n, :4]
        R = Rotation.from_quat([q[1], q[2], q[3], q[0]]).as_matrix()
        np.testing.assert_allclose(poses[n, 4:], W[name][:3, 3], atol=1e-6, err_msg=name)
        np.testing.assert_allclose(R, W[name][:3, :3], atol=1e-6, err_msg=name)


def test_file_path_and_errors(tmp_path):
    p = tmp_path / "r.urdf"
    p.write_text(URDF)
    assert load_urdf(str(p)).model.n_joints == 7
    bad = URDF.replace('<limit lower="-2" upper="2" velocity="1.5" effort="10"/>', "")
    with pytest.raises(ValueError, match="no limits"):
        load_urdf(bad)
