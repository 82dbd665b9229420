"""The URDF / SRDF loader on the spherized robots the reference ships
(``resources/*/*_spherized*.urdf``; skipped where the reference checkout is
absent): every link pose of the FP64 FK of the parsed model against an
independent 4x4 evaluation of the URDF, sphere counts per link, SRDF pair
removal, the reference's error on a joint without a velocity limit, and the
committed Panda fixture against a fresh parse."""

import math
import xml.etree.ElementTree as ET
from pathlib import Path

import numpy as np
import pytest
from scipy.spatial.transform import Rotation

from oracle import kinematics as okin
from oracle.refpath import reference_root
from pyroffi_b200.urdf import load_urdf, read_srdf_disabled_pairs

_REF = reference_root()
RES = _REF / "resources" if _REF is not None else Path("/nonexistent")
pytestmark = pytest.mark.skipif(not RES.is_dir(), reason="the reference checkout's resources are not present")
ROBOTS = sorted(str(p) for p in RES.glob("*/*_spherized*.urdf") if "ridgeback" not in p.name) if RES.is_dir() else []


def _floats(s, default):
    return np.array([float(v) for v in s.split()]) if s else np.array(default, float)


def matrix_fk(path, cfg, actuated):
    """link name -> 4x4 world transform, straight from the URDF XML."""
    root = ET.parse(path).getroot()
    joints = root.findall("joint")
    by_child = {j.find("child").get("link"): j for j in joints}
    act = {n: i for i, n in enumerate(actuated)}

    def q_of(j):
        name, m = j.get("name"), j.find("mimic")
        if name in act:
            return cfg[act[name]]
        if m is not None:
            base = cfg[act[m.get("joint")]] if m.get("joint") in act else 0.0
            return float(m.get("multiplier", 1.0)) * base + float(m.get("offset", 0.0))
        return 0.0

    W = {}

    def world(link):
        if link in W:
            return W[link]
        j = by_child.get(link)
        if j is None:
            W[link] = np.eye(4)
            return W[link]
        o = j.find("origin")
        T = np.eye(4)
        if o is not None:
            T[:3, :3] = Rotation.from_euler("xyz", _floats(o.get("rpy"), (0, 0, 0))).as_matrix()
            T[:3, 3] = _floats(o.get("xyz"), (0, 0, 0))
        axis = _floats(j.find("axis").get("xyz") if j.find("axis") is not None else None, (1, 0, 0))
        Mq = np.eye(4)
        q = q_of(j)
        if j.get("type") in ("revolute", "continuous"):
            Mq[:3, :3] = Rotation.from_rotvec(axis * q).as_matrix()
        elif j.get("type") == "prismatic":
            Mq[:3, 3] = axis * q
        W[link] = world(j.find("parent").get("link")) @ T @ Mq
        return W[link]

    return {l.get("name"): world(l.get("name")) for l in root.findall("link")}


@pytest.mark.parametrize("path", ROBOTS, ids=[Path(p).name for p in ROBOTS])
def test_fk_of_shipped_robot_matches_matrix_evaluation(path):
    r = load_urdf(path)
    rng = np.random.default_rng(len(path))
    lo, hi = r.model.lower.astype(np.float64), r.model.upper.astype(np.float64)
    for _ in range(3):
        cfg = rng.uniform(np.maximum(lo, -math.pi), np.minimum(hi, math.pi))
        poses = okin.forward_kinematics(cfg[None], r.model.as_dict())[0]
        W = matrix_fk(path, cfg, r.actuated_names)
        for n, name in enumerate(r.link_names):
            q = poses[n, :4]
            R = Rotation.from_quat([q[1], q[2], q[3], q[0]]).as_matrix()
            np.testing.assert_allclose(poses[n, 4:], W[name][:3, 3], atol=2e-5, err_msg=name)
            np.testing.assert_allclose(R, W[name][:3, :3], atol=2e-5, err_msg=name)


@pytest.mark.parametrize("path", ROBOTS, ids=[Path(p).name for p in ROBOTS])
def test_sphere_counts_per_link(path):
    r = load_urdf(path)
    root = ET.parse(path).getroot()
    for n, link in enumerate(root.findall("link")):
        want = sum(1 for c in link.findall("collision") if c.find("geometry") is not None
                   and c.find("geometry").find("sphere") is not None)
        assert int((r.spheres.radii[n] >= 0).sum()) == want, link.get("name")


def test_srdf_pairs_are_removed():
    urdf, srdf = RES / "panda" / "panda_spherized.urdf", RES / "panda" / "panda.srdf"
    r = load_urdf(str(urdf), srdf=str(srdf))
    idx = {n: k for k, n in enumerate(r.link_names)}
    pairs = {tuple(p) for p in r.active_pairs}
    for a, b in read_srdf_disabled_pairs(str(srdf)):
        if a in idx and b in idx:
            assert (max(idx[a], idx[b]), min(idx[a], idx[b])) not in pairs


def test_joint_without_velocity_limit_is_rejected_as_by_the_reference():
    # ridgeback's continuous wheel joints have no <limit>; the reference's
    # _get_joint_limit_vel raises on them too
    with pytest.raises(ValueError, match="velocity"):
        load_urdf(str(RES / "ridgeback" / "ridgeback_spherized.urdf"))


def test_committed_panda_fixture_is_current():
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from make_robot_fixtures import panda_arrays

    fresh = panda_arrays(RES.parent)
    z = np.load(Path(__file__).resolve().parent / "golden" / "robots" / "panda.npz")
    for k, v in fresh.items():
        np.testing.assert_array_equal(z[k], v, err_msg=k)
