"""The kernels on a robot loaded from URDF text: FK, the fused FK ->
sphere -> distance kernel and a few LM iterations against the FP64 oracle."""

import numpy as np
import pytest
import torch

from oracle import kinematics as okin
from oracle import lm as olm
from oracle import se3
from error_report import assert_distances
from pyroffi_b200 import workloads as W
from pyroffi_b200.collision import fk_sphere_collision
from pyroffi_b200.device import DeviceRobot, DeviceSpheres, DeviceWorld
from pyroffi_b200.ik import BatchIkSolver
from pyroffi_b200.urdf import load_urdf
from test_urdf import URDF

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def tt(x):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float32, device=DEV)


def test_fused_kernel_on_urdf_robot():
    r = load_urdf(URDF)
    m = r.model
    rng = np.random.default_rng(3)
    cfg = rng.uniform(m.lower, m.upper, size=(300, m.n_act)).astype(np.float32)
    world = W.empty_world()
    world.spheres = W.random_sphere_world(rng, 40)
    res = fk_sphere_collision(DeviceRobot.upload(m, DEV), DeviceSpheres.upload(r.spheres, DEV),
                              DeviceWorld.upload(world, DEV), tt(cfg), per_link=True)
    links = okin.forward_kinematics(cfg.astype(np.float64), m.as_dict())
    lp = res.link_poses.cpu().numpy()
    assert np.abs(lp[..., 4:] - links[..., 4:]).max() < 1e-5
    rel = se3.quat_mul(se3.quat_conj(lp[..., :4].astype(np.float64)), links[..., :4])
    assert se3.rotation_angle(rel).max() < 1e-5
    # per-link minimum distance to every obstacle sphere, padding skipped
    c = se3.apply(links[:, :, None, :], r.spheres.centers.astype(np.float64))       # [B, N, S, 3]
    d = np.linalg.norm(c[:, :, :, None, :] - world.spheres[None, None, None, :, :3], axis=-1)
    d = d - r.spheres.radii[None, :, :, None] - world.spheres[None, None, None, :, 3]
    d = np.where(r.spheres.radii[None, :, :, None] < 0, np.inf, d).min(axis=2)
    want = np.where(np.isinf(d), 1e9, d)
    assert_distances(res.dist_bnm.cpu().numpy(), want, quantity="signed distance (fused, per link)",
                     case="URDF robot")


@pytest.mark.parametrize("max_iter", [1, 2])
def test_lm_on_urdf_robot(max_iter):
    r = load_urdf(URDF)
    m = r.model
    tool = r.link_index("tool")
    rng = np.random.default_rng(5)
    tgt_cfg = rng.uniform(m.lower, m.upper, size=(2, m.n_act))
    Tj = okin.forward_kinematics(tgt_cfg, m.as_dict())[:, tool]
    seeds = rng.uniform(m.lower, m.upper, size=(2, 24, m.n_act)).astype(np.float32)
    s = BatchIkSolver(m, tool, max_iter=max_iter, lambda_init=1e-2, device=DEV)
    cfgs, errs = s.run_lm(tt(Tj[:, None, :]), tt(seeds))
    cfgs, errs = cfgs.cpu().numpy(), errs.cpu().numpy()
    ok = 0
    for p in range(2):
        oc, oe = olm.ls_ik(seeds[p], Tj[p][None, None], m.as_dict(), [m.link_joint(tool)],
                           [m.ancestor_mask(tool)], lower=m.lower, upper=m.upper, max_iter=max_iter,
                           lambda_init=1e-2, lambda_down=0.5, lambda_up=3.0, enable_collision=False)
        close = (np.abs(cfgs[p] - oc).max(axis=1) < 2e-4) & (np.abs(errs[p] - oe) <= 1e-3 * np.abs(oe) + 1e-4)
        ok += int(close.sum())
    assert ok >= 0.9 * 48, ok
