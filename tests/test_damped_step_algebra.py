"""The algebra behind the kernels' damped step (``csrc/pk_damped_step.cuh``),
restated in FP64 numpy and checked on random systems:

* the dual (Woodbury) form with a diagonal prior and held columns equals the
  primal system it replaces, ``(Js_F^T Js_F + diag(lam + pd_F)) x_F =
  -(Js_F^T (fw + Js_N xn_N) + v_F)``, ``x_N = xn_N``;
* with fewer free columns than rows the dual system is rank-deficient (its
  smallest eigenvalue is lam), while the primal one keeps the eigenvalues of
  ``Js_F^T Js_F`` + lam, and the reverse with more free columns than rows:
  the reason the kernels solve the smaller of the two."""

import numpy as np


def primal(J, fw, lam, pd, fr, xn, v):
    F, N = np.where(fr)[0], np.where(~fr)[0]
    f2 = fw + J[:, N] @ xn[N]
    A = J[:, F].T @ J[:, F] + np.diag(lam + pd[F])
    x = xn.copy()
    x[F] = np.linalg.solve(A, -(J[:, F].T @ f2 + v[F]))
    return x


def dual(J, fw, lam, pd, fr, xn, v):
    d = lam + pd
    w = np.where(fr, lam / d, 0.0)
    u = np.where(fr, v / d, -xn)
    M = (J * w) @ J.T + lam * np.eye(J.shape[0])
    z = np.linalg.solve(M, fw - J @ u)
    return np.where(fr, -u - w * (J.T @ z), xn)


def random_case(rng, R, n, n_free, prior):
    J = rng.normal(size=(R, n))
    fr = np.zeros(n, bool)
    fr[rng.choice(n, n_free, replace=False)] = True
    xn = np.where(fr, 0.0, rng.normal(size=n))
    pd = np.abs(rng.normal(size=n)) * 1e-3 if prior else np.zeros(n)
    v = rng.normal(size=n) * 1e-3 if prior else np.zeros(n)
    return J, rng.normal(size=R), pd, fr, xn, v


def test_dual_equals_primal():
    rng = np.random.default_rng(0)
    for R, n in ((6, 8), (12, 16)):
        for trial in range(100):
            n_free = int(rng.integers(R, n + 1))       # the dual form's domain: free columns >= rows
            J, fw, pd, fr, xn, v = random_case(rng, R, n, n_free, prior=trial % 2 == 1)
            lam = 10.0 ** rng.uniform(-4, 0)
            a, b = primal(J, fw, lam, pd, fr, xn, v), dual(J, fw, lam, pd, fr, xn, v)
            np.testing.assert_allclose(b, a, rtol=1e-8, atol=1e-10 * np.abs(a).max())


def test_held_columns_keep_their_values():
    rng = np.random.default_rng(1)
    J, fw, pd, fr, xn, v = random_case(rng, 6, 8, 6, prior=False)
    x = dual(J, fw, 1e-3, pd, fr, xn, v)
    np.testing.assert_array_equal(x[~fr], xn[~fr])


def test_the_smaller_system_is_the_well_conditioned_one():
    rng = np.random.default_rng(2)
    lam = 1e-8
    for n_free, dual_bad in ((7, False), (4, True)):
        J, _, _, fr, _, _ = random_case(rng, 6, 8, n_free, prior=False)
        JF = J[:, fr]
        ev_dual = np.linalg.eigvalsh(JF @ JF.T + lam * np.eye(6))
        ev_primal = np.linalg.eigvalsh(JF.T @ JF + lam * np.eye(n_free))
        if dual_bad:   # fewer free columns than rows: the dual carries the null space of Js_F^T
            assert ev_dual.min() < 10 * lam and ev_primal.min() > 1e3 * lam
        else:          # more free columns than rows: the primal carries the null space of Js_F
            assert ev_primal.min() < 10 * lam and ev_dual.min() > 1e3 * lam
