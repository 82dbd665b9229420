"""Shared cases of the per-seed IK kernel tests (HJCD, SQP): device tensors,
the agreement rate of two error arrays, and a two-EE robot problem."""

import numpy as np
import torch

from oracle import kinematics as okin
from pyroffi_b200 import workloads as W
from pyroffi_b200.hjcd import HjcdSolver

DEV = "cuda:0"


def t(a, dt=torch.float32):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=DEV)


def bimanual(P=3, S=32, seed=7, target_links=None, solver=HjcdSolver):
    """The 15-DOF two-arm tree; targets at its two hands, or at `target_links`
    (three or four EEs take the kernels' 4-EE variant)."""
    cl = W.mixed_classes()[2]
    m = cl.model
    tl = tuple(cl.target_links if target_links is None else target_links)
    rng = np.random.default_rng(seed)
    cfg = m.random_cfgs(rng, P)
    links = okin.forward_kinematics(cfg.astype(np.float64), m.as_dict())
    tgt = np.stack([links[:, l] for l in tl], axis=1).astype(np.float32)    # [P, n_ee, 7]
    seeds = rng.uniform(m.lower, m.upper, size=(P, S, m.n_act)).astype(np.float32)
    sol = solver(m, tl, device=DEV)
    tj = [m.link_joint(l) for l in tl]
    anc = [m.ancestor_mask(l) for l in tl]
    return m, sol, tj, anc, tgt, seeds


def agree(a, b, rtol=1e-3, atol=1e-7):
    return float(np.mean(np.abs(a - b) <= rtol * np.abs(b) + atol))
