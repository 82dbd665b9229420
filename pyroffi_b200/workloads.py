"""Seeded synthetic workloads of the five benchmark configurations.

Every array is drawn from ``numpy.random.default_rng(seed)``; nothing is read
from disk.  The shapes and distributions stand in for the reference's
URDF robots, ``bench_env*.json`` scenes and trajectory problems:

1. ``fk_collision`` (seed 1001): 7-DOF revolute chain, 8 spheres per moving
   link (56), 64 obstacle spheres, B configurations.
2. ``ik`` (seed 1002): same chain, 256 targets = FK of random in-limit
   configurations, 128 uniform seeds each, 100 obstacle spheres, 200
   self-collision sphere pairs between non-adjacent links.
3. ``trajectories`` (seed 1003): 512 x 64 x 7 trajectories (linear
   start->goal interpolation + N(0, 0.1) noise, endpoints kept), 256 obstacle
   spheres + 32 axis-aligned boxes.
4. ``mixed_ik`` (seed 1004): 4096 problems over four robot classes.
5. ``sweep`` (seed 1005): 7-DOF chain, 16 spheres per link, 4096 obstacle
   spheres + 256 oriented boxes.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .robot import RobotModel, RobotSpheres, random_spheres, serial_chain, bimanual_tree, humanoid_tree


@dataclass
class World:
    spheres: np.ndarray     # [Ms, 4]
    capsules: np.ndarray    # [Mc, 7]
    boxes: np.ndarray       # [Mb, 15]
    halfspaces: np.ndarray  # [Mh, 6]

    @property
    def M(self) -> int:
        return sum(a.shape[0] for a in (self.spheres, self.capsules, self.boxes, self.halfspaces))

    def arrays(self):
        return self.spheres, self.capsules, self.boxes, self.halfspaces


def empty_world() -> World:
    z = lambda k: np.zeros((0, k), np.float32)  # noqa: E731
    return World(z(4), z(7), z(15), z(6))


def random_sphere_world(rng, n, lo=-1.0, hi=1.0, r_range=(0.05, 0.2)) -> np.ndarray:
    c = rng.uniform(lo, hi, size=(n, 3))
    r = rng.uniform(*r_range, size=(n, 1))
    return np.concatenate([c, r], axis=1).astype(np.float32)


def random_boxes(rng, n, oriented: bool, half_range=(0.05, 0.3)) -> np.ndarray:
    """[n, 15]: centre U[-1,1]^3, axis columns of a random (or identity)
    rotation, half-lengths U[half_range]^3 (``_cuda_collision.py:148-156``)."""
    out = np.zeros((n, 15), np.float32)
    out[:, 0:3] = rng.uniform(-1, 1, size=(n, 3))
    for i in range(n):
        if oriented:
            q = rng.normal(size=4)
            q /= np.linalg.norm(q)
            w, x, y, z = q
            R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                          [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                          [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        else:
            R = np.eye(3)
        out[i, 3:6], out[i, 6:9], out[i, 9:12] = R[:, 0], R[:, 1], R[:, 2]
    out[:, 12:15] = rng.uniform(*half_range, size=(n, 3))
    return out


def self_sphere_pairs(link_of: np.ndarray, model: RobotModel, n_pairs: int, rng) -> np.ndarray:
    """n_pairs distinct (i, j) robot-sphere pairs, i < j, between links that
    are neither equal nor parent/child."""
    adj = set()
    for li in range(model.n_links):
        j = model.link_joint(li)
        if j < 0:
            continue
        p = int(model.parent_idx[j])
        # link li's parent link is the child link of joint p (link p+1 when links
        # are numbered base + one per joint), or the base link for root joints
        parent_link = int(np.nonzero(model.parent_joint_indices == p)[0][0]) if p >= 0 else \
            int(np.nonzero(model.parent_joint_indices == -1)[0][0])
        adj.add((min(li, parent_link), max(li, parent_link)))
    cand = [(i, j) for i in range(len(link_of)) for j in range(i + 1, len(link_of))
            if link_of[i] != link_of[j]
            and (min(link_of[i], link_of[j]), max(link_of[i], link_of[j])) not in adj]
    pick = rng.choice(len(cand), size=min(n_pairs, len(cand)), replace=False)
    return np.asarray([cand[k] for k in sorted(pick)], np.int32).reshape(-1, 2)


def active_link_pairs(model: RobotModel, spheres: RobotSpheres) -> np.ndarray:
    """Link pairs (i > j) to check for self-collision: both links carry
    spheres, not the same link, not parent/child (``_robot_collision.py:648-695``)."""
    has = (spheres.radii > 0).any(axis=1)
    adj = set()
    for li in range(model.n_links):
        j = model.link_joint(li)
        if j < 0:
            continue
        p = int(model.parent_idx[j])
        pl = int(np.nonzero(model.parent_joint_indices == p)[0][0]) if p >= 0 else \
            int(np.nonzero(model.parent_joint_indices == -1)[0][0])
        adj.add((max(li, pl), min(li, pl)))
    out = [(i, j) for i in range(model.n_links) for j in range(i)
           if has[i] and has[j] and (i, j) not in adj]
    return np.asarray(out, np.int32).reshape(-1, 2)


@dataclass
class FkCollisionWorkload:
    model: RobotModel
    spheres: RobotSpheres
    world: World
    cfg: np.ndarray  # [B, n_act]


def fk_collision(B: int = 1024, seed: int = 1001) -> FkCollisionWorkload:
    rng = np.random.default_rng(seed)
    model = serial_chain(7, rng)
    spheres = random_spheres(model, rng, per_link=8)
    world = empty_world()
    world.spheres = random_sphere_world(rng, 64)
    cfg = model.random_cfgs(rng, B)
    return FkCollisionWorkload(model, spheres, world, cfg)


def _quat_mul(a, b):
    w1, x1, y1, z1 = np.moveaxis(a, -1, 0)
    w2, x2, y2, z2 = np.moveaxis(b, -1, 0)
    return np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], -1)


def _quat_rot(q, v):
    t = 2.0 * np.cross(q[..., 1:4], v)
    return v + q[..., :1] * t + np.cross(q[..., 1:4], t)


def _scene_fk(model: RobotModel, cfg: np.ndarray) -> np.ndarray:
    """FP64 joint poses [B, n_j, 7] of revolute / prismatic / fixed joints.

    Used only to draw a feasible synthetic scene (target poses, obstacle
    rejection); no operator of this package calls it."""
    cfg = np.asarray(cfg, np.float64)
    B = cfg.shape[0]
    T = np.zeros((B, model.n_joints, 7))
    for j in model.topo_inv:
        src = model.mimic_act_idx[j] if model.mimic_act_idx[j] >= 0 else model.act_idx[j]
        q = (cfg[:, src] if src >= 0 else 0.0) * model.mimic_mul[j] + model.mimic_off[j]
        v, w = model.twists[j, :3].astype(np.float64), model.twists[j, 3:].astype(np.float64)
        q = np.broadcast_to(q, (B,))
        if np.any(w):
            assert not np.any(v), "screw joints are not used by the synthetic robots"
            nw = np.linalg.norm(w)
            half = 0.5 * q * nw
            qd = np.concatenate([np.cos(half)[:, None], np.sin(half)[:, None] * (w / nw)], -1)
            td = np.zeros((B, 3))
        else:
            qd = np.tile([1.0, 0, 0, 0], (B, 1))
            td = np.outer(np.broadcast_to(q, (B,)), v)
        ptf = model.parent_tf[j].astype(np.float64)
        q_pc = _quat_mul(ptf[None, :4], qd)
        t_pc = _quat_rot(np.broadcast_to(ptf[:4], (B, 4)), td) + ptf[4:]
        p = model.parent_idx[j]
        if p < 0:
            T[:, j, :4], T[:, j, 4:] = q_pc, t_pc
        else:
            T[:, j, :4] = _quat_mul(T[:, p, :4], q_pc)
            T[:, j, 4:] = _quat_rot(T[:, p, :4], t_pc) + T[:, p, 4:]
    return T


@dataclass
class IkWorkload:
    model: RobotModel
    spheres: RobotSpheres
    world: World
    target_link: int
    target_cfgs: np.ndarray     # [P, n_act] configurations the targets come from
    target_T: np.ndarray        # [P, 7] EE target poses (FK of target_cfgs), float32
    seeds: np.ndarray           # [P, Sd, n_act]
    spheres_local: np.ndarray   # [n_rs, 4]
    sphere_joint: np.ndarray    # [n_rs]
    self_pairs: np.ndarray      # [n_self, 2]
    max_iter: int = 30
    lambda_init: float = 1e-2
    lambda_down: float = 0.1
    lambda_up: float = 10.0
    pos_weight: float = 50.0
    ori_weight: float = 10.0
    collision_weight: float = 1e4
    collision_margin: float = 0.02
    pos_tol: float = 1e-3
    rot_tol: float = 1e-2


def _sphere_world(model: RobotModel, rs, jidx, cfg):
    T = _scene_fk(model, cfg)[:, jidx]                       # [B, n_rs, 7]
    return _quat_rot(T[..., :4], rs[None, :, :3].astype(np.float64)) + T[..., 4:]


def ik(P: int = 256, Sd: int = 128, seed: int = 1002, n_obstacles: int = 100, n_self: int = 200,
       target_spread: float = 0.6, clearance: float = 0.03) -> IkWorkload:
    """Feasible collision-aware IK problems.

    Targets are FK of random in-limit configurations drawn within
    +-target_spread rad of a self-collision-free nominal posture and kept
    only when free of all ``n_self`` self pairs; obstacle spheres (centres
    U[-1,1]^3, radius U[0.05,0.2]) are kept only when every robot sphere at
    every target configuration clears them by ``clearance`` (> the 0.02 m
    margin).  So every target is reachable without penalty, while seeds,
    uniform over the full limits, start mostly elsewhere and often in
    collision.  (Uniform targets in a uniform 100-sphere field are nearly
    never collision-free, which would make the 1 mm success criterion
    unreachable for any solver.)
    """
    rng = np.random.default_rng(seed)
    model = serial_chain(7, rng)
    spheres = random_spheres(model, rng, per_link=8)
    rs, jidx, link_of = spheres.flat_for_ik(model)
    pairs = self_sphere_pairs(link_of, model, n_self, rng)
    margin = 0.02

    def self_free(cfg):
        p = _sphere_world(model, rs, jidx, cfg)
        d = np.linalg.norm(p[:, pairs[:, 0]] - p[:, pairs[:, 1]], axis=-1) - (rs[pairs[:, 0], 3] + rs[pairs[:, 1], 3])
        return np.all(d > clearance, axis=-1) if len(pairs) else np.ones(len(cfg), bool)

    while True:
        nominal = model.random_cfgs(rng, 1)
        if self_free(nominal)[0]:
            break
    targets = []
    while len(targets) < P:
        c = np.clip(nominal + rng.uniform(-target_spread, target_spread, size=(max(64, 2 * P), model.n_act)),
                    model.lower, model.upper).astype(np.float32)
        targets.extend(c[self_free(c)])
    target_cfgs = np.asarray(targets[:P], np.float32)
    occupied = _sphere_world(model, rs, jidx, target_cfgs).reshape(-1, 3)
    occ_r = np.tile(rs[:, 3], P)
    obs = []
    while len(obs) < n_obstacles:
        o = np.concatenate([rng.uniform(-1.0, 1.0, 3), rng.uniform(0.05, 0.2, 1)])
        if np.min(np.linalg.norm(occupied - o[:3], axis=-1) - (occ_r + o[3])) > clearance:
            obs.append(o)
    world = empty_world()
    world.spheres = np.asarray(obs, np.float32).reshape(-1, 4)
    tj = model.link_joint(model.n_links - 1)
    target_T = _scene_fk(model, target_cfgs)[:, tj].astype(np.float32)
    seeds = rng.uniform(model.lower, model.upper, size=(P, Sd, model.n_act)).astype(np.float32)
    assert margin < clearance
    return IkWorkload(model=model, spheres=spheres, world=world, target_link=model.n_links - 1,
                      target_cfgs=target_cfgs, target_T=target_T, seeds=seeds, spheres_local=rs,
                      sphere_joint=jidx, self_pairs=pairs)


@dataclass
class TrajWorkload:
    model: RobotModel
    spheres: RobotSpheres
    world: World
    traj: np.ndarray            # [Bt, T, n_act]
    link_pairs: np.ndarray      # [P, 2] active self link pairs (i > j)
    margin: float = 0.01
    w_smooth: float = 1.0
    w_acc: float = 0.5
    w_jerk: float = 0.1
    w_limits: float = 1.0
    w_collision: float = 3.0


def trajectories(Bt: int = 512, T: int = 64, seed: int = 1003) -> TrajWorkload:
    rng = np.random.default_rng(seed)
    model = serial_chain(7, rng)
    spheres = random_spheres(model, rng, per_link=8)
    world = empty_world()
    world.spheres = random_sphere_world(rng, 256)
    world.boxes = random_boxes(rng, 32, oriented=False)
    start = model.random_cfgs(rng, Bt)
    goal = model.random_cfgs(rng, Bt)
    s = np.linspace(0.0, 1.0, T)[None, :, None]
    traj = start[:, None, :] * (1 - s) + goal[:, None, :] * s
    noise = rng.normal(0.0, 0.1, size=traj.shape)
    noise[:, 0] = 0.0
    noise[:, -1] = 0.0
    traj = (traj + noise).astype(np.float32)
    return TrajWorkload(model, spheres, world, traj, active_link_pairs(model, spheres))


def random_capsules(rng, n, length=(0.1, 0.5), r_range=(0.03, 0.1)) -> np.ndarray:
    """[n, 7]: (p1, p2, r) with p1 U[-1,1]^3 and p2 = p1 + a random direction times U[length]."""
    p1 = rng.uniform(-1, 1, size=(n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    p2 = p1 + d * rng.uniform(*length, size=(n, 1))
    r = rng.uniform(*r_range, size=(n, 1))
    return np.concatenate([p1, p2, r], axis=1).astype(np.float32)


def mixed_trajectories(Bt: int = 4, T: int = 16, seed: int = 1006, n_spheres: int = 24, n_capsules: int = 6,
                       n_boxes: int = 6, per_link: int = 4) -> TrajWorkload:
    """Trajectories of the 7-DOF chain among all four obstacle kinds (spheres,
    capsules, oriented boxes and a floor halfspace) -- the small SCO case."""
    rng = np.random.default_rng(seed)
    model = serial_chain(7, rng)
    spheres = random_spheres(model, rng, per_link=per_link)
    world = empty_world()
    world.spheres = random_sphere_world(rng, n_spheres)
    world.capsules = random_capsules(rng, n_capsules)
    world.boxes = random_boxes(rng, n_boxes, oriented=True)
    world.halfspaces = np.array([[0.0, 0.0, 1.0, 0.0, 0.0, -1.2]], np.float32)
    start = model.random_cfgs(rng, 1)[0]
    goal = model.random_cfgs(rng, 1)[0]
    s = np.linspace(0.0, 1.0, T)[None, :, None]
    traj = np.broadcast_to(start[None, None] * (1 - s) + goal[None, None] * s, (Bt, T, start.shape[0])).copy()
    noise = rng.normal(0.0, 0.05, size=traj.shape)
    noise[:, 0] = 0.0
    noise[:, -1] = 0.0
    traj = (traj + noise).astype(np.float32)
    return TrajWorkload(model, spheres, world, traj, active_link_pairs(model, spheres))


@dataclass
class SweepWorkload:
    model: RobotModel
    spheres: RobotSpheres
    world: World
    cfg: np.ndarray


def sweep(B: int, seed: int = 1005) -> SweepWorkload:
    rng = np.random.default_rng(seed)
    model = serial_chain(7, rng)
    spheres = random_spheres(model, rng, per_link=16)
    world = empty_world()
    world.spheres = random_sphere_world(rng, 4096)
    world.boxes = random_boxes(rng, 256, oriented=True)
    cfg = model.random_cfgs(rng, B)
    return SweepWorkload(model, spheres, world, cfg)


@dataclass
class MixedIkClass:
    model: RobotModel
    spheres: RobotSpheres
    target_links: tuple
    fraction: float


def mixed_classes(seed: int = 1004) -> list[MixedIkClass]:
    rng = np.random.default_rng(seed)
    c7 = serial_chain(7, rng)
    c6 = serial_chain(6, rng)
    bi = bimanual_tree(rng)
    hu = humanoid_tree(rng)
    return [
        MixedIkClass(c7, random_spheres(c7, rng, per_link=8), (c7.n_links - 1,), 0.4),
        MixedIkClass(c6, random_spheres(c6, rng, per_link=8), (c6.n_links - 1,), 0.3),
        MixedIkClass(bi, random_spheres(bi, rng, per_link=8), (10, 16), 0.2),
        MixedIkClass(hu, random_spheres(hu, rng, per_link_range=(4, 12)), (10, 17), 0.1),
    ]


@dataclass
class MixedIkWorkload:
    """Uneven IK batch: problems of several robot classes sharing one world."""
    classes: list                 # [MixedIkClass]
    world: World
    problem_class: np.ndarray     # [P] class of each problem
    n_seeds: np.ndarray           # [P] seeds of each problem
    target_T: list                # per class [P_c, n_ee, 7] float32 (problems of that class, in order)
    target_cfgs: list             # per class [P_c, n_act]
    seeds: list                   # per class [P_c, max seeds of the class, n_act] (unused slots 0)
    index_in_class: np.ndarray    # [P] position of problem p within its class
    max_iter: int = 30
    lambda_init: float = 1e-2
    lambda_down: float = 0.1
    lambda_up: float = 10.0
    pos_weight: float = 50.0
    ori_weight: float = 10.0
    collision_weight: float = 1e4
    collision_margin: float = 0.02
    pos_tol: float = 1e-3
    rot_tol: float = 1e-2


def mixed_ik(n_problems: int = 4096, seed: int = 1004, n_obstacles: int = 500, seeds_range=(32, 256),
             target_spread: float = 0.6, clearance: float = 0.03) -> MixedIkWorkload:
    """Mixed persistent-batch IK: 40% 7-DOF chain, 30% 6-DOF chain, 20% 15-DOF
    bimanual tree (two hand targets), 10% 29-DOF humanoid (two hand targets),
    U{32..256} seeds per problem, 500 obstacle spheres.

    As in ``ik``, each class's targets are FK of configurations within
    +-target_spread rad of one nominal posture, and obstacle spheres (centres
    U[-1.5,1.5]^3, radius U[0.05,0.2]) are kept only when every sphere of every
    target configuration clears them by ``clearance``; seeds are uniform over
    the joint limits.
    """
    from scipy.spatial import cKDTree

    classes = mixed_classes(seed)
    rng = np.random.default_rng(seed + 7)
    fr = np.array([c.fraction for c in classes])
    counts = np.floor(fr * n_problems).astype(int)
    counts[0] += n_problems - counts.sum()
    problem_class = np.repeat(np.arange(len(classes)), counts)
    rng.shuffle(problem_class)
    n_seeds = rng.integers(seeds_range[0], seeds_range[1] + 1, size=n_problems)
    index_in_class = np.zeros(n_problems, np.int64)
    for c in range(len(classes)):
        idx = np.nonzero(problem_class == c)[0]
        index_in_class[idx] = np.arange(len(idx))
    target_T, target_cfgs, seeds, occupied, occ_r = [], [], [], [], []
    for c, cl in enumerate(classes):
        m = cl.model
        Pc = int(counts[c])
        nominal = m.random_cfgs(rng, 1)
        cfgs = np.clip(nominal + rng.uniform(-target_spread, target_spread, size=(Pc, m.n_act)),
                       m.lower, m.upper).astype(np.float32)
        Tj = _scene_fk(m, cfgs)
        tj = [m.link_joint(l) for l in cl.target_links]
        target_T.append(Tj[:, tj].astype(np.float32))
        target_cfgs.append(cfgs)
        rs, jidx, _ = cl.spheres.flat_for_ik(m)
        occupied.append(_sphere_world(m, rs, jidx, cfgs).reshape(-1, 3))
        occ_r.append(np.tile(rs[:, 3], Pc))
        sd = int(n_seeds[problem_class == c].max()) if Pc else 0
        seeds.append(rng.uniform(m.lower, m.upper, size=(Pc, sd, m.n_act)).astype(np.float32))
    occupied = np.concatenate(occupied)
    occ_r = np.concatenate(occ_r)
    tree = cKDTree(occupied)
    r_max = float(occ_r.max())
    obs = []
    while len(obs) < n_obstacles:
        o = np.concatenate([rng.uniform(-1.5, 1.5, 3), rng.uniform(0.05, 0.2, 1)])
        near = tree.query_ball_point(o[:3], o[3] + r_max + clearance)
        if not near or np.min(np.linalg.norm(occupied[near] - o[:3], axis=-1) - (occ_r[near] + o[3])) > clearance:
            obs.append(o)
    world = empty_world()
    world.spheres = np.asarray(obs, np.float32).reshape(-1, 4)
    return MixedIkWorkload(classes=classes, world=world, problem_class=problem_class, n_seeds=n_seeds,
                           target_T=target_T, target_cfgs=target_cfgs, seeds=seeds,
                           index_in_class=index_in_class)
