"""Pin the FP64 oracle to the reference's own helper code (golden vectors
recorded by tests/golden/make_golden.py from the reference's CUDA helper
headers compiled for the host).  The reference runs in FP32, so tolerances
are FP32-sized."""

import numpy as np
import pytest

from oracle import collision as oc
from oracle import kinematics as okin
from oracle import lm as olm
from oracle import se3

ROBOTS = ["chain7", "bimanual15", "humanoid29", "odd6"]


def test_se3_exp(golden):
    """Revolute (v = 0) and prismatic (omega = 0) motions -- the only ones a
    URDF joint produces -- match the reference helper.  For screw tangents the
    reference CUDA helper (_fk_cuda_helpers.cuh:123-130) computes
    A v + B w x v + C w x (w x v) with A = sin t / t, i.e. jaxlie's
    V v = v + B w x v + C w x (w x v) plus (A - 1) v; the oracle follows jaxlie
    (the reference's JAX path), and this test pins that exact difference."""
    tang = golden["se3_exp_in"].astype(np.float64)
    out = se3.exp(tang)
    ref = golden["se3_exp_out"].astype(np.float64)
    np.testing.assert_allclose(out[:32], ref[:32], atol=2e-6, rtol=1e-5)
    th = np.linalg.norm(tang[32:, 3:], axis=-1)
    A = np.sin(th) / th
    expected_ref = out[32:].copy()
    expected_ref[:, 4:] += (A - 1.0)[:, None] * tang[32:, :3]
    np.testing.assert_allclose(expected_ref, ref[32:], atol=5e-6, rtol=1e-5)


def test_se3_compose(golden):
    out = se3.compose(golden["se3_compose_a"].astype(np.float64), golden["se3_compose_b"].astype(np.float64))
    np.testing.assert_allclose(out, golden["se3_compose_out"], atol=2e-6, rtol=1e-5)


@pytest.mark.parametrize("name", ROBOTS)
def test_fk_matches_reference(golden, name):
    g = lambda k: golden[f"fk_{name}_{k}"]  # noqa: E731
    topo = okin.topo_sort(g("parent_idx"))
    np.testing.assert_array_equal(topo, g("topo_inv"))
    T = okin.fk_joints(g("cfg"), g("twists"), g("parent_tf"), g("parent_idx"), g("act_idx"),
                       g("mimic_mul"), g("mimic_off"), g("mimic_act_idx"), topo)
    ref = g("out").astype(np.float64)
    # quaternion sign is fixed by the composition, no flip needed
    np.testing.assert_allclose(T[..., 4:], ref[..., 4:], atol=1e-5)
    np.testing.assert_allclose(T[..., :4], ref[..., :4], atol=1e-5)


@pytest.mark.parametrize("name", ["chain7", "bimanual15", "odd6"])
def test_residual_jacobian_matches_reference(golden, name):
    g = lambda k: golden[f"fk_{name}_{k}"]  # noqa: E731
    h = lambda k: golden[f"resjac_{name}_{k}"]  # noqa: E731
    model = dict(twists=g("twists"), parent_tf=g("parent_tf"), parent_idx=g("parent_idx"),
                 act_idx=g("act_idx"), mimic_mul=g("mimic_mul"), mimic_off=g("mimic_off"),
                 mimic_act_idx=g("mimic_act_idx"), topo_inv=g("topo_inv"),
                 n_act=h("cfg").shape[1], n_joints=g("twists").shape[0])
    Tj = olm._fk(h("cfg"), model)
    r, J = olm.residual_and_jacobian(Tj, h("target_jnts"), h("target").astype(np.float64), model,
                                     h("ancestor_masks"))
    np.testing.assert_allclose(r, h("r"), atol=2e-5, rtol=1e-4)
    np.testing.assert_allclose(J, h("J"), atol=2e-5, rtol=1e-4)


@pytest.mark.parametrize("n", [7, 15])
def test_cholesky_matches_reference(golden, n):
    A, b, x, ok = golden[f"chol{n}_A"], golden[f"chol{n}_b"], golden[f"chol{n}_x"], golden[f"chol{n}_ok"]
    out = olm.chol_solve(A.copy(), b.copy())
    np.testing.assert_array_equal(ok == 0, np.all(out == 0, axis=-1))
    np.testing.assert_allclose(out, x, rtol=1e-9, atol=1e-9 * np.abs(x).max())


def test_distance_primitives_match_reference(golden):
    g = golden
    s, s2, c, c2, b, h = (g[k].astype(np.float64) for k in
                          ("dist_sph", "dist_sph2", "dist_cap", "dist_cap2", "dist_box", "dist_hs"))
    tol = dict(atol=3e-6, rtol=1e-5)
    np.testing.assert_allclose(oc.sphere_sphere(s[:, :3], s[:, 3], s2[:, :3], s2[:, 3]), g["dist_ss"], **tol)
    np.testing.assert_allclose(oc.sphere_capsule(s[:, :3], s[:, 3], c[:, :3], c[:, 3:6], c[:, 6]), g["dist_sc"], **tol)
    np.testing.assert_allclose(oc.sphere_box(s[:, :3], s[:, 3], b), g["dist_sb"], **tol)
    np.testing.assert_allclose(oc.sphere_halfspace(s[:, :3], s[:, 3], h), g["dist_sh"], **tol)
    np.testing.assert_allclose(oc.capsule_capsule(c[:, :3], c[:, 3:6], c[:, 6], c2[:, :3], c2[:, 3:6], c2[:, 6]),
                               g["dist_cc"], atol=2e-5, rtol=1e-4)
    np.testing.assert_allclose(oc.capsule_box(c[:, :3], c[:, 3:6], c[:, 6], b), g["dist_cb"], atol=2e-5, rtol=1e-4)
    np.testing.assert_allclose(oc.capsule_halfspace(c[:, :3], c[:, 3:6], c[:, 6], h), g["dist_ch"], **tol)


def test_colldist_from_sdf_matches_reference(golden):
    np.testing.assert_allclose(oc.colldist_from_sdf(golden["colldist_in"].astype(np.float64), 0.02),
                               golden["colldist_out"], atol=1e-7, rtol=1e-5)
