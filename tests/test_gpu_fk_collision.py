"""GPU parity: FK, collision drop-ins and the fused FK->collision kernel
against the FP64 oracle (tolerances: FK 1e-5 m / 1e-5 rad, sphere centres
1e-5 m, distances 1e-5 m).  Each test records the largest error it saw
(``error_report``)."""

import numpy as np
import pytest
import torch

from oracle import collision as oc
from oracle import kinematics as okin
from oracle import se3
from pyroffi_b200 import robot as R
from pyroffi_b200 import workloads as W
from pyroffi_b200.collision import fk_sphere_collision
from pyroffi_b200.cuda_kernels import (collision_self_capsule, collision_self_sphere,
                                       collision_world_capsule, collision_world_sphere,
                                       collision_world_sphere_reduced, fk_cuda)
from pyroffi_b200.device import DeviceRobot, DeviceSpheres, DeviceWorld
from error_report import assert_distances, record

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
POS_TOL = 1e-5
ROT_TOL = 1e-5


def tt(x, dtype=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=DEV)


def rot_angle(q1, q2):
    rel = se3.quat_mul(se3.quat_conj(q1.astype(np.float64)), q2.astype(np.float64))
    return se3.rotation_angle(rel)


def oracle_fk(model_like, cfg):
    g = model_like
    return okin.fk_joints(cfg, g["twists"], g["parent_tf"], g["parent_idx"], g["act_idx"], g["mimic_mul"],
                          g["mimic_off"], g["mimic_act_idx"], g["topo_inv"])


def run_fk(g, cfg):
    starts, joints, _ = okin.fk_depth_schedule(g["parent_idx"], g["topo_inv"])
    out = fk_cuda(tt(cfg), tt(g["twists"]), tt(g["parent_tf"]), tt(g["parent_idx"], torch.int32),
                  tt(g["act_idx"], torch.int32), tt(g["mimic_mul"]), tt(g["mimic_off"]),
                  tt(g["mimic_act_idx"], torch.int32), tt(g["topo_inv"], torch.int32),
                  tt(starts, torch.int32), tt(joints, torch.int32))
    return out.cpu().numpy()


@pytest.mark.parametrize("name", ["chain7", "bimanual15", "humanoid29", "odd6"])
@pytest.mark.parametrize("B", [1, 16, 129, 4096])
def test_fk_cuda_matches_oracle(golden, name, B):
    g = {k: golden[f"fk_{name}_{k}"] for k in ("twists", "parent_tf", "parent_idx", "act_idx", "mimic_mul",
                                                "mimic_off", "mimic_act_idx", "topo_inv", "lower", "upper")}
    rng = np.random.default_rng(B)
    cfg = rng.uniform(g["lower"], g["upper"], size=(B, len(g["lower"]))).astype(np.float32)
    out = run_fk(g, cfg)
    ref = oracle_fk(g, cfg)
    assert out.shape == ref.shape
    pe, re = np.abs(out[..., 4:] - ref[..., 4:]).max(), rot_angle(out[..., :4], ref[..., :4]).max()
    record("FK joint position (fk_cuda)", pe, f"{name} B={B}", "m")
    record("FK joint rotation (fk_cuda)", re, f"{name} B={B}", "rad")
    assert pe < POS_TOL
    assert re < ROT_TOL


def test_fk_cuda_reproduces_reference_golden(golden):
    """The golden FK outputs recorded from the reference's own fk_single."""
    for name in ("chain7", "bimanual15", "humanoid29", "odd6"):
        g = {k: golden[f"fk_{name}_{k}"] for k in ("twists", "parent_tf", "parent_idx", "act_idx", "mimic_mul",
                                                    "mimic_off", "mimic_act_idx", "topo_inv")}
        out = run_fk(g, golden[f"fk_{name}_cfg"])
        ref = golden[f"fk_{name}_out"]
        assert np.abs(out[..., 4:] - ref[..., 4:]).max() < POS_TOL
        assert rot_angle(out[..., :4], ref[..., :4]).max() < ROT_TOL


def test_fk_cuda_batch_axes_and_empty(golden):
    g = {k: golden[f"fk_chain7_{k}"] for k in ("twists", "parent_tf", "parent_idx", "act_idx", "mimic_mul",
                                                "mimic_off", "mimic_act_idx", "topo_inv")}
    starts, joints, _ = okin.fk_depth_schedule(g["parent_idx"], g["topo_inv"])
    args = [tt(g["twists"]), tt(g["parent_tf"]), tt(g["parent_idx"], torch.int32), tt(g["act_idx"], torch.int32),
            tt(g["mimic_mul"]), tt(g["mimic_off"]), tt(g["mimic_act_idx"], torch.int32),
            tt(g["topo_inv"], torch.int32), tt(starts, torch.int32), tt(joints, torch.int32)]
    cfg = torch.rand((2, 3, 7), device=DEV)
    assert fk_cuda(cfg, *args).shape == (2, 3, 7, 7)
    assert fk_cuda(torch.zeros((0, 7), device=DEV), *args).shape == (0, 7, 7)


# ---------------------------------------------------------------------------
# collision drop-ins
# ---------------------------------------------------------------------------

def mixed_world(rng, Ms=37, Mc=5, Mb=6, Mh=3):
    ws = W.random_sphere_world(rng, Ms)
    wc = np.concatenate([rng.uniform(-1, 1, (Mc, 6)), rng.uniform(0.02, 0.1, (Mc, 1))], 1).astype(np.float32)
    wb = W.random_boxes(rng, Mb, oriented=True)
    n = rng.normal(size=(Mh, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    wh = np.concatenate([n, rng.uniform(-1, 1, (Mh, 3))], 1).astype(np.float32)
    return ws, wc, wb, wh


def sphere_robot_batch(rng, B, S, N, pad_frac=0.2):
    c = rng.uniform(-1, 1, size=(B, S, N, 3)).astype(np.float32)
    r = rng.uniform(0.02, 0.1, size=(B, S, N)).astype(np.float32)
    r[rng.uniform(size=r.shape) < pad_frac] = -1e9
    return c, r


@pytest.mark.parametrize("world_kind", ["mixed", "spheres_only", "empty", "m_mult4"])
def test_world_sphere_and_reduced(world_kind):
    rng = np.random.default_rng(11)
    B, S, N = 33, 4, 6
    K = S * N
    c_bsn, r_bsn = sphere_robot_batch(rng, B, S, N)
    # SoA [3, B, K] with k = s*N + n
    centers = np.ascontiguousarray(c_bsn.reshape(B, K, 3).transpose(2, 0, 1))
    radii = r_bsn.reshape(B, K)
    if world_kind == "mixed":
        world = mixed_world(rng)
    elif world_kind == "spheres_only":
        world = (W.random_sphere_world(rng, 45), np.zeros((0, 7), np.float32), np.zeros((0, 15), np.float32),
                 np.zeros((0, 6), np.float32))
    elif world_kind == "m_mult4":
        world = mixed_world(rng, Ms=8, Mc=4, Mb=2, Mh=2)
    else:
        world = (np.zeros((0, 4), np.float32), np.zeros((0, 7), np.float32), np.zeros((0, 15), np.float32),
                 np.zeros((0, 6), np.float32))
    wt = [tt(x) for x in world]
    out = collision_world_sphere(tt(centers), tt(radii), *wt).cpu().numpy()
    ref = oc.world_sphere(c_bsn.reshape(B, K, 3).astype(np.float64), radii, *[x.astype(np.float64) for x in world])
    assert out.shape == ref.shape
    assert_distances(out, ref, quantity="signed distance (collision_world_sphere)", case=world_kind)
    red = collision_world_sphere_reduced(tt(centers), tt(radii), *wt, n=N).cpu().numpy()
    rref = oc.world_sphere_reduced(c_bsn.reshape(B, K, 3).astype(np.float64), radii,
                                   *[x.astype(np.float64) for x in world], N)
    assert red.shape == rref.shape
    assert_distances(red, rref, quantity="signed distance (collision_world_sphere_reduced)", case=world_kind)


def test_world_capsule_robot():
    rng = np.random.default_rng(12)
    B, N = 19, 5
    caps = np.concatenate([rng.uniform(-1, 1, (B, N, 6)), rng.uniform(0.02, 0.1, (B, N, 1))], -1).astype(np.float32)
    caps[0, 0, 3:6] = caps[0, 0, 0:3]                      # degenerate segment
    world = mixed_world(rng)
    soa = np.ascontiguousarray(caps.transpose(2, 0, 1))    # [7, B, N]
    out = collision_world_capsule(tt(soa), *[tt(x) for x in world]).cpu().numpy()
    ws, wc, wb, wh = (x.astype(np.float64) for x in world)
    c = caps.astype(np.float64)[:, :, None, :]
    ref = np.concatenate([
        oc.sphere_capsule(ws[:, :3], ws[:, 3], c[..., 0:3], c[..., 3:6], c[..., 6]),
        oc.capsule_capsule(c[..., 0:3], c[..., 3:6], c[..., 6], wc[:, 0:3], wc[:, 3:6], wc[:, 6]),
        oc.capsule_box(c[..., 0:3], c[..., 3:6], c[..., 6], wb),
        oc.capsule_halfspace(c[..., 0:3], c[..., 3:6], c[..., 6], wh)], axis=-1)
    assert_distances(out, ref, quantity="signed distance (collision_world_capsule)")


def test_self_sphere_and_capsule():
    rng = np.random.default_rng(13)
    B, S, N = 21, 5, 7
    c, r = sphere_robot_batch(rng, B, S, N, pad_frac=0.3)
    pairs = np.array([(i, j) for i in range(N) for j in range(i)], np.int32)
    out = collision_self_sphere(tt(c), tt(r), tt(pairs[:, 0], torch.int32), tt(pairs[:, 1], torch.int32)).cpu().numpy()
    ref = oc.self_sphere_full(c.astype(np.float64), r.astype(np.float64), pairs[:, 0], pairs[:, 1])
    assert_distances(out, ref, quantity="signed distance (collision_self_sphere)")
    caps = np.concatenate([rng.uniform(-1, 1, (B, N, 6)), rng.uniform(0.02, 0.1, (B, N, 1))], -1).astype(np.float32)
    out = collision_self_capsule(tt(caps), tt(pairs[:, 0], torch.int32), tt(pairs[:, 1], torch.int32)).cpu().numpy()
    c64 = caps.astype(np.float64)
    ref = oc.capsule_capsule(c64[:, pairs[:, 0], 0:3], c64[:, pairs[:, 0], 3:6], c64[:, pairs[:, 0], 6],
                             c64[:, pairs[:, 1], 0:3], c64[:, pairs[:, 1], 3:6], c64[:, pairs[:, 1], 6])
    assert_distances(out, ref, quantity="signed distance (collision_self_capsule)")
    empty = collision_self_sphere(tt(c), tt(r), tt(np.zeros(0), torch.int32), tt(np.zeros(0), torch.int32))
    assert empty.shape == (B, 0)


# ---------------------------------------------------------------------------
# fused FK -> spheres -> distances
# ---------------------------------------------------------------------------

def fused_reference(model, spheres, world, cfg):
    md = model.as_dict()
    Tj = oracle_fk(md, cfg)
    links = okin.link_poses(Tj, model.parent_joint_indices)                       # [B,N,7]
    c = se3.apply(links[:, :, None, :], spheres.centers.astype(np.float64))        # [B,N,S,3]
    B, N, S = c.shape[:3]
    c_k = np.swapaxes(c, 1, 2).reshape(B, S * N, 3)                                # k = s*N + n
    r_k = np.broadcast_to(spheres.radii.T.reshape(-1), (B, S * N))
    bkm = oc.world_sphere(c_k, r_k, *[x.astype(np.float64) for x in world.arrays()])
    valid = r_k >= 0
    dmin = np.where(valid[..., None], bkm, np.inf).min(axis=(1, 2))
    return links, bkm, np.minimum(dmin, 1e9)


@pytest.mark.parametrize("case", ["config1", "tree_mixed"])
def test_fused_fk_sphere_collision(case):
    if case == "config1":
        w = W.fk_collision(B=1024)
        model, spheres, world, cfg = w.model, w.spheres, w.world, w.cfg
    else:
        rng = np.random.default_rng(3)
        model = R.bimanual_tree(rng)
        spheres = R.random_spheres(model, rng, per_link_range=(2, 6))
        world = W.empty_world()
        world.spheres, world.capsules, world.boxes, world.halfspaces = mixed_world(rng, Ms=21, Mc=3, Mb=4, Mh=2)
        cfg = model.random_cfgs(rng, 77)
    res = fk_sphere_collision(DeviceRobot.upload(model, DEV), DeviceSpheres.upload(spheres, DEV),
                              DeviceWorld.upload(world, DEV), tt(cfg), per_sphere=True, sphere_centers=True)
    links, bkm, dmin = fused_reference(model, spheres, world, cfg)
    lp = res.link_poses.cpu().numpy()
    pe, re = np.abs(lp[..., 4:] - links[..., 4:]).max(), rot_angle(lp[..., :4], links[..., :4]).max()
    record("FK link position (fused)", pe, case, "m")
    record("FK link rotation (fused)", re, case, "rad")
    assert pe < POS_TOL
    assert re < ROT_TOL
    # sphere centres (at_config), k = s*N + n, compared directly
    c = se3.apply(links[:, :, None, :], spheres.centers.astype(np.float64))     # [B,N,S,3]
    B, N, S = c.shape[:3]
    ck = np.swapaxes(c, 1, 2).reshape(B, S * N, 3)
    sc = res.sphere_centers.cpu().numpy()
    cerr = np.abs(sc[..., :3] - ck).max()
    record("sphere centre (fused, at_config)", cerr, case, "m")
    assert cerr < POS_TOL
    np.testing.assert_array_equal(sc[..., 3], np.broadcast_to(spheres.radii.T.reshape(-1), (B, S * N)))
    assert_distances(res.dist_bkm.cpu().numpy(), bkm, quantity="signed distance (fused, per sphere)", case=case)
    assert_distances(res.min_dist.cpu().numpy(), dmin, quantity="signed distance (fused, minimum)", case=case)


def test_fused_large_batch_min_only():
    w = W.fk_collision(B=65536 + 17)
    res = fk_sphere_collision(DeviceRobot.upload(w.model, DEV), DeviceSpheres.upload(w.spheres, DEV),
                              DeviceWorld.upload(w.world, DEV), tt(w.cfg), link_poses=False)
    idx = np.random.default_rng(0).choice(len(w.cfg), 512, replace=False)
    _, _, dmin = fused_reference(w.model, w.spheres, w.world, w.cfg[idx])
    assert_distances(res.min_dist.cpu().numpy()[idx], dmin, quantity="signed distance (fused, minimum)",
                     case="65553 configs")


@pytest.mark.parametrize("both", [False, True])
@pytest.mark.parametrize("case", ["sweep", "padded"])
def test_fused_per_link_rows(case, both):
    """[B, N, M] per-link rows (the reduced layout) from the fused kernel, alone or with [B, K, M]."""
    if case == "sweep":
        w = W.sweep(B=24)     # 16 spheres per link, 4096 spheres + 256 boxes
        model, spheres, world, cfg = w.model, w.spheres, w.world, w.cfg
    else:
        rng = np.random.default_rng(5)
        model = R.bimanual_tree(rng)
        spheres = R.random_spheres(model, rng, per_link_range=(0, 5))
        world = W.empty_world()
        world.spheres, world.capsules, world.boxes, world.halfspaces = mixed_world(rng, Ms=9, Mc=5, Mb=3, Mh=1)
        cfg = model.random_cfgs(rng, 45)
    res = fk_sphere_collision(DeviceRobot.upload(model, DEV), DeviceSpheres.upload(spheres, DEV),
                              DeviceWorld.upload(world, DEV), tt(cfg), per_sphere=both, per_link=True)
    links, bkm, dmin = fused_reference(model, spheres, world, cfg)
    B, N, S = len(cfg), spheres.n_links, spheres.S
    r_k = np.broadcast_to(spheres.radii.T.reshape(-1), (B, S * N))
    d = np.where(r_k[..., None] < 0, np.inf, bkm).reshape(B, S, N, -1).min(axis=1)
    bnm = np.where(np.isinf(d), 1e9, d)
    assert_distances(res.dist_bnm.cpu().numpy(), bnm, quantity="signed distance (fused, per link)", case=case)
    assert_distances(res.min_dist.cpu().numpy(), dmin, quantity="signed distance (fused, minimum)", case=case)
    if both:
        assert_distances(res.dist_bkm.cpu().numpy(), bkm, quantity="signed distance (fused, per sphere)", case=case)


@pytest.mark.parametrize("case", ["sweep", "padded"])
def test_per_link_rows_identical_with_and_without_per_sphere_rows(case):
    """The per-link pass reads the link-pair centre layout; with per-sphere rows
    requested too, the centres are rewritten in pairs after that pass.  Both
    routes must give the same bits."""
    if case == "sweep":
        w = W.sweep(B=40)
        model, spheres, world, cfg = w.model, w.spheres, w.world, w.cfg
    else:
        rng = np.random.default_rng(8)
        model = R.bimanual_tree(rng)
        spheres = R.random_spheres(model, rng, per_link_range=(0, 5))
        world = W.empty_world()
        world.spheres, world.capsules, world.boxes, world.halfspaces = mixed_world(rng, Ms=13, Mc=2, Mb=5, Mh=1)
        cfg = model.random_cfgs(rng, 33)
    args = (DeviceRobot.upload(model, DEV), DeviceSpheres.upload(spheres, DEV), DeviceWorld.upload(world, DEV),
            tt(cfg))
    a = fk_sphere_collision(*args, per_sphere=False, per_link=True)
    b = fk_sphere_collision(*args, per_sphere=True, per_link=True)
    assert torch.equal(a.dist_bnm, b.dist_bnm)


def test_no_world_staging_wait_gave_up():
    """Kernels that copy the world into shared memory with the TMA engine wait
    for it with a bound; a block that gives up is counted.  After staged
    launches of the fused kernel and the trajectory kernel, the count is 0."""
    import ctypes as C
    from pyroffi_b200 import _lib
    from pyroffi_b200.trajopt import TrajectoryCost
    w = W.fk_collision(B=256)
    fk_sphere_collision(DeviceRobot.upload(w.model, DEV), DeviceSpheres.upload(w.spheres, DEV),
                        DeviceWorld.upload(w.world, DEV), tt(w.cfg), per_sphere=True)
    wt = W.trajectories(Bt=8, T=16)
    TrajectoryCost(wt.model, wt.spheres, wt.world, wt.link_pairs, margin=wt.margin, device=DEV).cost_and_grad(
        torch.as_tensor(wt.traj, device=DEV))
    torch.cuda.synchronize()
    n = C.c_uint64(123)
    assert _lib.load().pk_stage_wait_timeouts(C.byref(n)) == _lib.PK_OK
    assert n.value == 0


def test_forced_staging_timeout_is_reported_and_results_are_unchanged():
    """The bounded wait's test hook: with force_timeout set, no TMA copy is
    issued, every staging block waits out a 0.2 ms limit (by the GPU's global
    timer), counts itself and loads the obstacle arrays plainly.  The host
    then reads PK_ERR_TIMEOUT, and the outputs (fused collision, trajectory
    cost and gradient, LM IK) equal the normal path's bit for bit.  Nothing
    is in flight at any point, and the hook is switched off again whatever
    happens."""
    import ctypes as C
    from pyroffi_b200 import _lib
    from pyroffi_b200.trajopt import TrajectoryCost
    lib = _lib.load()
    w = W.fk_collision(B=300)
    args = (DeviceRobot.upload(w.model, DEV), DeviceSpheres.upload(w.spheres, DEV),
            DeviceWorld.upload(w.world, DEV), tt(w.cfg))
    wt = W.trajectories(Bt=8, T=16)
    tc = TrajectoryCost(wt.model, wt.spheres, wt.world, wt.link_pairs, margin=wt.margin, device=DEV)
    x = torch.as_tensor(wt.traj, device=DEV)
    from pyroffi_b200.ik import BatchIkSolver
    wi = W.ik(P=4, Sd=64)
    lm = BatchIkSolver(wi.model, wi.target_link, spheres=wi.spheres, world=wi.world, self_pairs=wi.self_pairs,
                       max_iter=3, lambda_init=wi.lambda_init, lambda_down=wi.lambda_down, lambda_up=wi.lambda_up,
                       device=DEV)
    tg, sd = tt(wi.target_T), tt(wi.seeds)

    def run():
        r = fk_sphere_collision(*args, per_sphere=True)
        c, g = tc.cost_and_grad(x)
        q, e = lm.run_lm(tg, sd)
        torch.cuda.synchronize()
        return r.min_dist.clone(), r.dist_bkm.clone(), c.clone(), g.clone(), q.clone(), e.clone()

    n = C.c_uint64(0)
    assert lib.pk_stage_wait_reset() == _lib.PK_OK
    normal = run()
    assert lib.pk_stage_wait_timeouts(C.byref(n)) == _lib.PK_OK and n.value == 0
    try:
        assert lib.pk_stage_wait_configure(1, 200_000) == _lib.PK_OK
        forced = run()
    finally:
        assert lib.pk_stage_wait_configure(0, 0) == _lib.PK_OK
    assert lib.pk_stage_wait_timeouts(C.byref(n)) == _lib.PK_ERR_TIMEOUT
    assert n.value >= 2, n.value              # at least one block of each kernel
    assert b"gave up" in lib.pk_last_error() and b"untrusted" not in lib.pk_last_error()
    for a, b in zip(normal, forced):
        assert torch.equal(a, b)
    assert lib.pk_stage_wait_reset() == _lib.PK_OK
    after = run()
    assert lib.pk_stage_wait_timeouts(C.byref(n)) == _lib.PK_OK and n.value == 0
    for a, b in zip(normal, after):
        assert torch.equal(a, b)
