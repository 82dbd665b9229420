"""CHOMP oracle math on the CPU: the metric operator equals its dense
pentadiagonal matrix, and the truncated CG solves it when run to
convergence."""

import numpy as np
from oracle import chomp as ochomp


def test_metric_apply_is_pentadiagonal():
    n, reg = 9, 1e-3
    A = np.zeros((n, n))
    for i in range(n):
        for j, v in ((i, 6.0 + reg), (i - 1, -4.0), (i + 1, -4.0), (i - 2, 1.0), (i + 2, 1.0)):
            if 0 <= j < n:
                A[i, j] = v
    x = np.random.default_rng(0).normal(size=(3, n))
    got = np.stack([ochomp.metric_apply(xi, reg) for xi in x])
    np.testing.assert_allclose(got, x @ A.T, rtol=1e-12, atol=1e-12)


def test_cg_solves_the_metric():
    n, reg = 20, 1e-3
    b = np.random.default_rng(1).normal(size=n)
    x = ochomp.cg_solve(b.copy(), reg, 200, 1e-14)
    # the reference's +1e-9 in the step-length denominators bounds the attainable residual
    np.testing.assert_allclose(ochomp.metric_apply(x, reg), b, rtol=1e-5, atol=1e-5)
