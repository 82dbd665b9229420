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


def bimanual(P=3, S=32, seed=7):
    cl = W.mixed_classes()[2]
    m = cl.model
    rng = np.random.default_rng(seed)
    cfg = m.random_cfgs(rng, P)
    links = okin.forward_kinematics(cfg.astype(np.float64), m.as_dict())
    tgt = np.stack([links[:, l] for l in cl.target_links], axis=1).astype(np.float32)    # [P, 2, 7]
    seeds = rng.uniform(m.lower, m.upper, size=(P, S, m.n_act)).astype(np.float32)
    sol = HjcdSolver(m, cl.target_links, device=DEV)
    tj = [m.link_joint(l) for l in cl.target_links]
    anc = [m.ancestor_mask(l) for l in cl.target_links]
    return m, sol, tj, anc, tgt, seeds


def agree(a, b, rtol=1e-3, atol=1e-7):
    return float(np.mean(np.abs(a - b) <= rtol * np.abs(b) + atol))
