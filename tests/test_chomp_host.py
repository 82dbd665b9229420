"""CHOMP host math on CPU tensors: the metric operator equals its dense
pentadiagonal matrix, and the batched truncated CG equals the oracle's
per-timeline CG (same iteration count and stopping rule)."""

import numpy as np
import torch

from oracle import chomp as ochomp
from pyroffi_b200.chomp import cg_solve, metric_apply


def test_metric_apply_is_pentadiagonal():
    n, reg = 9, 1e-3
    A = np.zeros((n, n))
    for i in range(n):
        for j, v in ((i, 6.0 + reg), (i - 1, -4.0), (i + 1, -4.0), (i - 2, 1.0), (i + 2, 1.0)):
            if 0 <= j < n:
                A[i, j] = v
    x = np.random.default_rng(0).normal(size=(3, n))
    got = metric_apply(torch.as_tensor(x), reg).numpy()
    np.testing.assert_allclose(got, x @ A.T, rtol=1e-12, atol=1e-12)


def test_batched_cg_equals_oracle_cg():
    rng = np.random.default_rng(1)
    b = rng.normal(size=(6, 30))
    b[2] *= 1e-9  # stops after its first step
    got = cg_solve(torch.as_tensor(b), 1e-3, 24, 1e-4).numpy()
    for i in range(6):
        np.testing.assert_allclose(got[i], ochomp.cg_solve(b[i].copy(), 1e-3, 24, 1e-4), rtol=1e-9, atol=1e-15)
