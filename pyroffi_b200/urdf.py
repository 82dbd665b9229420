"""URDF / SRDF -> robot model, collision spheres and self-collision link pairs.

Restates, on the standard-library XML parser, what the reference builds from
a ``yourdfpy.URDF``:

* ``RobotURDFParser.parse`` (``src/pyroffi/_robot_urdf_parser.py:270-412``):
  joints and links in document order; a joint is *actuated* when it is not
  fixed and not a mimic; twists ``[0, axis]`` (revolute / continuous) and
  ``[axis, 0]`` (prismatic), zero otherwise (``:455-471``); parent
  transforms from ``<origin xyz rpy>`` as wxyz_xyz (``:473-497``); the parent
  joint is the joint whose child is this joint's parent link; limits of the
  actuated joints, continuous joints without limits get [-pi, pi]
  (``:499-531``); a mimic of an actuated joint takes its multiplier / offset,
  a mimic of a non-actuated joint is fixed (``:414-453``); link -> parent
  joint indices; a parent-first topological order that also puts a mimicked
  joint before its mimic (``:147-218``) and the FK depth schedule.
* ``RobotCollisionSpherized.from_urdf`` (``collision/_robot_collision.py:446-581``):
  each link's ``<collision>`` spheres (centre = the collision origin's
  translation, radius as given; other geometry is skipped), padded to the
  largest count with radius -1e9.
* the active self-collision pairs (``:583-695``): all (i, j) with i > j in
  ``tril_indices`` order, minus the diagonal, minus parent/child links of a
  joint (``ignore_immediate_adjacents``) and user pairs -- or, when an SRDF is
  given, minus only its ``<disable_collisions>`` pairs
  (``_robot_srdf_parser.py``).

Mesh and primitive collision geometry other than spheres is not
converted (the reference warns and skips it as well).
"""

from __future__ import annotations

import math
import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass

import numpy as np

from .robot import PAD_RADIUS, RobotModel, RobotSpheres, depth_schedule


@dataclass
class UrdfRobot:
    model: RobotModel
    spheres: RobotSpheres
    joint_names: tuple
    actuated_names: tuple
    link_names: tuple
    active_pairs: np.ndarray        # [P, 2] link index pairs (i, j), i > j
    velocity_limits: np.ndarray     # [n_act]
    lower_all: np.ndarray           # [n_joints]
    upper_all: np.ndarray
    base_link: str

    def link_index(self, name: str) -> int:
        return self.link_names.index(name)


def _floats(text, n, default):
    if text is None:
        return list(default)
    v = [float(x) for x in text.split()]
    if len(v) != n:
        raise ValueError(f"expected {n} numbers, got {text!r}")
    return v


def rpy_to_wxyz(r: float, p: float, y: float) -> np.ndarray:
    """Quaternion (w, x, y, z) of the URDF fixed-axis rotation Rz(y) Ry(p) Rx(r)."""
    cr, sr = math.cos(r / 2), math.sin(r / 2)
    cp, sp = math.cos(p / 2), math.sin(p / 2)
    cy, sy = math.cos(y / 2), math.sin(y / 2)
    return np.array([cy * cp * cr + sy * sp * sr, cy * cp * sr - sy * sp * cr,
                     cy * sp * cr + sy * cp * sr, sy * cp * cr - cy * sp * sr])


def _origin(elem):
    o = elem.find("origin") if elem is not None else None
    xyz = _floats(o.get("xyz") if o is not None else None, 3, (0.0, 0.0, 0.0))
    rpy = _floats(o.get("rpy") if o is not None else None, 3, (0.0, 0.0, 0.0))
    return xyz, rpy


def _root(source):
    if isinstance(source, (str, os.PathLike)) and not str(source).lstrip().startswith("<"):
        return ET.parse(source).getroot()
    return ET.fromstring(source)


def read_srdf_disabled_pairs(srdf) -> list:
    """(link1, link2) of every ``<disable_collisions>`` of an SRDF (path or text)."""
    return [(e.get("link1"), e.get("link2")) for e in _root(srdf).findall("disable_collisions")]


def read_srdf_group_states(srdf) -> dict:
    """{group: {state: {joint: value}}} from the SRDF's ``<group_state>`` entries."""
    out: dict = {}
    for e in _root(srdf).findall("group_state"):
        joints = {j.get("name"): float(j.get("value")) for j in e.findall("joint")}
        out.setdefault(e.get("group"), {})[e.get("name")] = joints
    return out


def load_urdf(source, *, srdf=None, user_ignore_pairs=(), ignore_immediate_adjacents: bool = True,
              name: str | None = None) -> UrdfRobot:
    """Parse a URDF (file path or XML text) into the kernels' robot arrays."""
    root = _root(source)
    links = [l.get("name") for l in root.findall("link")]
    joints = root.findall("joint")
    jnames = [j.get("name") for j in joints]
    jtype = [j.get("type") for j in joints]
    jparent = [j.find("parent").get("link") for j in joints]
    jchild = [j.find("child").get("link") for j in joints]
    mimic = []
    for j in joints:
        m = j.find("mimic")
        mimic.append(None if m is None else (m.get("joint"), float(m.get("multiplier", 1.0)),
                                             float(m.get("offset", 0.0))))
    actuated = [i for i, j in enumerate(joints) if jtype[i] != "fixed" and mimic[i] is None]
    act_of = {i: k for k, i in enumerate(actuated)}
    child_joint = {jchild[i]: i for i in range(len(joints))}
    children = set(jchild)
    roots = [l for l in links if l not in children]
    if len(roots) != 1:
        raise ValueError(f"URDF must have exactly one root link, found {roots}")

    nj = len(joints)
    twists = np.zeros((nj, 6))
    ptf = np.zeros((nj, 7))
    parent_idx = np.full(nj, -1, np.int32)
    act_idx = np.full(nj, -1, np.int32)
    mimic_act = np.full(nj, -1, np.int32)
    mul, off = np.ones(nj), np.zeros(nj)
    lower_all, upper_all = np.zeros(nj), np.zeros(nj)
    vel_all = np.zeros(nj)
    for i, j in enumerate(joints):
        axis = np.array(_floats(j.find("axis").get("xyz") if j.find("axis") is not None else None, 3,
                                (1.0, 0.0, 0.0)))
        if jtype[i] in ("revolute", "continuous"):
            twists[i, 3:] = axis
        elif jtype[i] == "prismatic":
            twists[i, :3] = axis
        xyz, rpy = _origin(j)
        ptf[i, :4] = rpy_to_wxyz(*rpy)
        ptf[i, 4:] = xyz
        parent_idx[i] = child_joint.get(jparent[i], -1)
        if mimic[i] is not None:
            target, mul[i], off[i] = mimic[i]
            if target not in jnames:
                raise ValueError(f"joint {jnames[i]!r} mimics unknown joint {target!r}")
            t = jnames.index(target)
            mimic_act[i] = act_of.get(t, -1)  # a mimic of a non-actuated joint is fixed
        elif i in act_of:
            act_idx[i] = act_of[i]
        lim = j.find("limit")
        if jtype[i] == "fixed":
            lo = hi = vel = 0.0
        else:
            lo = float(lim.get("lower")) if lim is not None and lim.get("lower") is not None else None
            hi = float(lim.get("upper")) if lim is not None and lim.get("upper") is not None else None
            vel = float(lim.get("velocity")) if lim is not None and lim.get("velocity") is not None else None
            if lo is None or hi is None:
                if jtype[i] != "continuous":
                    raise ValueError(f"joint {jnames[i]!r} ({jtype[i]}) has no limits")
                lo, hi = -math.pi, math.pi
            if vel is None:
                raise ValueError(f"joint {jnames[i]!r} ({jtype[i]}) has no velocity limit")
        lower_all[i], upper_all[i], vel_all[i] = lo, hi, vel
    parent_joint_indices = np.array([child_joint.get(l, -1) for l in links], np.int32)
    model = RobotModel(twists=twists, parent_tf=ptf, parent_idx=parent_idx, act_idx=act_idx, mimic_mul=mul,
                       mimic_off=off, mimic_act_idx=mimic_act, parent_joint_indices=parent_joint_indices,
                       lower=lower_all[actuated], upper=upper_all[actuated],
                       name=name or root.get("name", "robot"))
    # parent-first order in which a mimicked joint also precedes its mimic
    mimic_dep = [jnames.index(m[0]) if m is not None else -1 for m in mimic]
    placed, order, remaining = set(), [], list(range(nj))
    while remaining:
        for pos, i in enumerate(remaining):
            p = int(parent_idx[i])
            if (p < 0 or p in placed) and (mimic_dep[i] < 0 or mimic_dep[i] in placed):
                order.append(i)
                placed.add(i)
                remaining.pop(pos)
                break
        else:
            raise ValueError(f"joint graph has a cycle: {[jnames[i] for i in remaining]}")
    model.topo_inv = np.asarray(order, np.int32)
    model.fk_level_starts, model.fk_level_joints = depth_schedule(model.parent_idx, model.topo_inv)

    # collision spheres per link
    per_link = []
    for l in root.findall("link"):
        sph = []
        for c in l.findall("collision"):
            g = c.find("geometry")
            s = g.find("sphere") if g is not None else None
            if s is None:
                continue
            xyz, _ = _origin(c)
            sph.append((xyz, float(s.get("radius"))))
        per_link.append(sph)
    S = max(1, max((len(s) for s in per_link), default=0))
    centers = np.zeros((len(links), S, 3), np.float32)
    radii = np.full((len(links), S), PAD_RADIUS, np.float32)
    for n, sph in enumerate(per_link):
        for s, (xyz, r) in enumerate(sph):
            centers[n, s] = xyz
            radii[n, s] = r
    spheres = RobotSpheres(centers=centers, radii=radii)

    # active self-collision pairs
    idx = {l: k for k, l in enumerate(links)}
    ignore = np.eye(len(links), dtype=bool)
    if srdf is not None:
        ignored = read_srdf_disabled_pairs(srdf)
    else:
        ignored = list(user_ignore_pairs)
        if ignore_immediate_adjacents:
            ignored += list(zip(jparent, jchild))
    for a, b in ignored:
        if a in idx and b in idx:
            ignore[idx[a], idx[b]] = ignore[idx[b], idx[a]] = True
    ii, jj = np.tril_indices(len(links), k=-1)
    keep = ~ignore[ii, jj]
    pairs = np.stack([ii[keep], jj[keep]], axis=1).astype(np.int32)

    return UrdfRobot(model=model, spheres=spheres, joint_names=tuple(jnames),
                     actuated_names=tuple(jnames[i] for i in actuated), link_names=tuple(links),
                     active_pairs=pairs, velocity_limits=vel_all[actuated].astype(np.float32),
                     lower_all=lower_all.astype(np.float32), upper_all=upper_all.astype(np.float32),
                     base_link=roots[0])
