"""Robot description arrays and synthetic robots.

``RobotModel`` carries exactly the flat arrays of the reference's
``JointInfo`` / ``LinkInfo`` (``src/pyroffi/_robot_urdf_parser.py:15-69,131-137``)
that the kernels read: twists, parent transforms, parent / actuated / mimic
indices, the topological order ``_topo_sort_inv`` and the FK depth schedule
(``fk_level_starts`` / ``fk_level_joints``, computed as
``_compute_fk_depth_schedule``, ``:234-267``), link -> parent-joint indices and
the actuated joint limits.

Synthetic robots (no URDF files are read): serial revolute chains, a 15-DOF
mobile bimanual tree and a 29-DOF humanoid tree, all drawn from a seeded
``numpy.random.Generator``.  Collision spheres per link live in
``RobotSpheres`` in the reference's padded ``[N, S]`` layout (padding
radius -1e9, ``src/pyroffi/collision/_robot_collision.py:492-503``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

PAD_RADIUS = -1e9


def _unit(rng: np.random.Generator, n: int | None = None) -> np.ndarray:
    v = rng.normal(size=(3,) if n is None else (n, 3))
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def topo_sort(parent_idx) -> np.ndarray:
    """Parent-first joint order; the first ready joint is taken each round
    (``RobotURDFParser._topologically_sort_joints``, parent dependencies)."""
    parent_idx = [int(p) for p in parent_idx]
    remaining = list(range(len(parent_idx)))
    placed: set[int] = set()
    order: list[int] = []
    while remaining:
        for pos, j in enumerate(remaining):
            if parent_idx[j] == -1 or parent_idx[j] in placed:
                order.append(j)
                placed.add(j)
                remaining.pop(pos)
                break
        else:
            raise ValueError(f"joint graph has a cycle or a dangling parent: {remaining}")
    return np.asarray(order, np.int32)


def depth_schedule(parent_idx, topo_inv):
    """(level_starts[L+1], level_joints[n_j]) grouping joints by tree depth."""
    n = len(parent_idx)
    depth = np.zeros(n, np.int64)
    for j in topo_inv:
        p = int(parent_idx[int(j)])
        depth[int(j)] = 0 if p < 0 else depth[p] + 1
    L = int(depth.max()) + 1 if n else 1
    starts, joints = [0], []
    for d in range(L):
        joints.extend(int(j) for j in topo_inv if depth[int(j)] == d)
        starts.append(len(joints))
    return np.asarray(starts, np.int32), np.asarray(joints, np.int32)


@dataclass
class RobotModel:
    twists: np.ndarray            # [n_j, 6] float32, [v, omega]
    parent_tf: np.ndarray         # [n_j, 7] float32, wxyz_xyz
    parent_idx: np.ndarray        # [n_j] int32, -1 = root
    act_idx: np.ndarray           # [n_j] int32, -1 = not directly actuated
    mimic_mul: np.ndarray         # [n_j] float32
    mimic_off: np.ndarray         # [n_j] float32
    mimic_act_idx: np.ndarray     # [n_j] int32
    parent_joint_indices: np.ndarray  # [n_links] int32, -1 = base link
    lower: np.ndarray             # [n_act] float32
    upper: np.ndarray             # [n_act] float32
    name: str = "robot"
    topo_inv: np.ndarray = field(init=False)
    fk_level_starts: np.ndarray = field(init=False)
    fk_level_joints: np.ndarray = field(init=False)

    def __post_init__(self):
        f32 = lambda x: np.ascontiguousarray(x, dtype=np.float32)  # noqa: E731
        i32 = lambda x: np.ascontiguousarray(x, dtype=np.int32)  # noqa: E731
        self.twists, self.parent_tf = f32(self.twists), f32(self.parent_tf)
        self.mimic_mul, self.mimic_off = f32(self.mimic_mul), f32(self.mimic_off)
        self.lower, self.upper = f32(self.lower), f32(self.upper)
        self.parent_idx, self.act_idx = i32(self.parent_idx), i32(self.act_idx)
        self.mimic_act_idx, self.parent_joint_indices = i32(self.mimic_act_idx), i32(self.parent_joint_indices)
        self.topo_inv = topo_sort(self.parent_idx)
        self.fk_level_starts, self.fk_level_joints = depth_schedule(self.parent_idx, self.topo_inv)

    @property
    def n_joints(self) -> int:
        return int(self.twists.shape[0])

    @property
    def n_act(self) -> int:
        return int(self.lower.shape[0])

    @property
    def n_links(self) -> int:
        return int(self.parent_joint_indices.shape[0])

    @property
    def n_levels(self) -> int:
        return int(self.fk_level_starts.shape[0] - 1)

    def link_joint(self, link: int) -> int:
        return int(self.parent_joint_indices[link])

    def ancestor_mask(self, link: int) -> np.ndarray:
        """Joints on the path from the root to ``link``'s parent joint
        (``_ls_ik.py:1090-1102``)."""
        m = np.zeros(self.n_joints, np.int32)
        j = self.link_joint(link)
        while j >= 0:
            m[j] = 1
            j = int(self.parent_idx[j])
        return m

    def as_dict(self) -> dict:
        return dict(twists=self.twists, parent_tf=self.parent_tf, parent_idx=self.parent_idx,
                    act_idx=self.act_idx, mimic_mul=self.mimic_mul, mimic_off=self.mimic_off,
                    mimic_act_idx=self.mimic_act_idx, topo_inv=self.topo_inv,
                    parent_joint_indices=self.parent_joint_indices, n_act=self.n_act,
                    n_joints=self.n_joints, lower=self.lower, upper=self.upper)

    def random_cfgs(self, rng: np.random.Generator, n: int) -> np.ndarray:
        return rng.uniform(self.lower, self.upper, size=(n, self.n_act)).astype(np.float32)


@dataclass
class RobotSpheres:
    """Per-link collision spheres in link frames, padded to [N, S]."""

    centers: np.ndarray   # [N, S, 3] float32
    radii: np.ndarray     # [N, S] float32 (PAD_RADIUS = padding)

    @property
    def n_links(self) -> int:
        return int(self.centers.shape[0])

    @property
    def S(self) -> int:
        return int(self.centers.shape[1])

    def link_spheres(self) -> np.ndarray:
        """[N, S, 4] (x, y, z, r) as the fused kernel takes them."""
        return np.ascontiguousarray(np.concatenate([self.centers, self.radii[..., None]], -1), np.float32)

    def flat_for_ik(self, model: RobotModel):
        """(spheres_local [n_rs, 4], joint_idx [n_rs], link_of [n_rs]) in parent-joint
        frames, skipping base links and padding, link-major order as
        ``_prepare_ls_collision_buffers_uncached`` (``_ls_ik.py:113-130``)."""
        rs, jidx, link_of = [], [], []
        for li in range(min(self.n_links, model.n_links)):
            j = model.link_joint(li)
            if j < 0:
                continue
            for si in range(self.S):
                r = float(self.radii[li, si])
                if r <= 0.0:
                    continue
                rs.append([*self.centers[li, si], r])
                jidx.append(j)
                link_of.append(li)
        return (np.asarray(rs, np.float32).reshape(-1, 4), np.asarray(jidx, np.int32),
                np.asarray(link_of, np.int32))


def _revolute_joint_arrays(parents, axes, offsets, rots=None):
    n = len(parents)
    twists = np.zeros((n, 6), np.float32)
    twists[:, 3:] = axes
    ptf = np.zeros((n, 7), np.float32)
    ptf[:, 0] = 1.0
    if rots is not None:
        ptf[:, :4] = rots
    ptf[:, 4:] = offsets
    return twists, ptf


def serial_chain(n_dof: int, rng: np.random.Generator, offset_range=(0.05, 0.40), limit=2.8,
                 name: str | None = None) -> RobotModel:
    """Serial revolute chain: joint i has parent i-1, parent transform
    (identity rotation, L_i u_i) with L_i ~ U[offset_range], u_i and the
    joint axis uniform on S^2, limits +-limit.  Links: base + one per joint."""
    L = rng.uniform(*offset_range, size=n_dof)
    u = _unit(rng, n_dof)
    axes = _unit(rng, n_dof)
    twists, ptf = _revolute_joint_arrays(list(range(-1, n_dof - 1)), axes, L[:, None] * u)
    return RobotModel(
        twists=twists, parent_tf=ptf, parent_idx=np.arange(-1, n_dof - 1),
        act_idx=np.arange(n_dof), mimic_mul=np.ones(n_dof), mimic_off=np.zeros(n_dof),
        mimic_act_idx=-np.ones(n_dof), parent_joint_indices=np.arange(-1, n_dof),
        lower=-limit * np.ones(n_dof), upper=limit * np.ones(n_dof),
        name=name or f"chain{n_dof}")


def _tree(rng, spec, name):
    """spec: list of (parent_joint, kind, axis or None) with kind in
    {'rev','pris','fixed'}; offsets drawn U[0.05,0.35] along random dirs."""
    n = len(spec)
    twists = np.zeros((n, 6), np.float32)
    ptf = np.zeros((n, 7), np.float32)
    ptf[:, 0] = 1.0
    parent = np.zeros(n, np.int32)
    act = -np.ones(n, np.int32)
    lower, upper = [], []
    a = 0
    for j, (p, kind, axis) in enumerate(spec):
        parent[j] = p
        ax = np.asarray(axis, np.float64) if axis is not None else _unit(rng)
        if p >= 0 or kind != "pris":
            ptf[j, 4:] = rng.uniform(0.05, 0.35) * _unit(rng)
        if kind == "rev":
            twists[j, 3:] = ax
        elif kind == "pris":
            twists[j, :3] = ax
        if kind != "fixed":
            act[j] = a
            a += 1
            lo, hi = (-1.5, 1.5) if kind == "pris" else (-2.8, 2.8)
            lower.append(lo)
            upper.append(hi)
    return RobotModel(twists=twists, parent_tf=ptf, parent_idx=parent, act_idx=act,
                      mimic_mul=np.ones(n), mimic_off=np.zeros(n), mimic_act_idx=-np.ones(n),
                      parent_joint_indices=np.arange(-1, n), lower=np.asarray(lower),
                      upper=np.asarray(upper), name=name)


def bimanual_tree(rng: np.random.Generator) -> RobotModel:
    """15-DOF mobile bimanual tree: prismatic x, prismatic y, revolute z
    (planar base), a fixed torso joint, then two 6-DOF revolute arms
    branching from the torso.  16 joints, 17 links; EE links 10 and 16."""
    spec = [(-1, "pris", (1, 0, 0)), (0, "pris", (0, 1, 0)), (1, "rev", (0, 0, 1)), (2, "fixed", None)]
    for _arm in range(2):
        prev = 3
        for _ in range(6):
            spec.append((prev, "rev", None))
            prev = len(spec) - 1
    return _tree(rng, spec, "bimanual15")


def humanoid_tree(rng: np.random.Generator) -> RobotModel:
    """29-DOF humanoid tree rooted at the pelvis: a 3-DOF waist chain to the
    torso, two 7-DOF arms from the torso, two 6-DOF legs from the pelvis.
    29 revolute joints, 30 links; hands are links 10 and 17."""
    spec = [(-1, "rev", None), (0, "rev", None), (1, "rev", None)]  # waist -> torso (joint 2)
    for _arm in range(2):
        prev = 2
        for _ in range(7):
            spec.append((prev, "rev", None))
            prev = len(spec) - 1
    for _leg in range(2):
        prev = -1
        for _ in range(6):
            spec.append((prev, "rev", None))
            prev = len(spec) - 1
    return _tree(rng, spec, "humanoid29")


def random_spheres(model: RobotModel, rng: np.random.Generator, per_link=8, per_link_range=None,
                   center_half=0.05, radius_range=(0.03, 0.08), base_spheres=False) -> RobotSpheres:
    """Spheres per moving link: centre U[-center_half, center_half]^3 in the link
    frame, radius U[radius_range]; ``per_link_range=(lo, hi)`` draws a count per
    link; base links get padding only unless ``base_spheres``."""
    N = model.n_links
    counts = np.full(N, per_link)
    if per_link_range is not None:
        counts = rng.integers(per_link_range[0], per_link_range[1] + 1, size=N)
    if not base_spheres:
        counts[model.parent_joint_indices < 0] = 0
    S = max(1, int(counts.max()))
    centers = np.zeros((N, S, 3), np.float32)
    radii = np.full((N, S), PAD_RADIUS, np.float32)
    for n in range(N):
        c = int(counts[n])
        centers[n, :c] = rng.uniform(-center_half, center_half, size=(c, 3))
        radii[n, :c] = rng.uniform(*radius_range, size=c)
    return RobotSpheres(centers=centers, radii=radii)
