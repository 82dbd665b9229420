"""CPU oracle for the pyroffi kinematics hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product path (``pyroffi_b200``)
never imports, links or executes anything under ``oracle/``, and fails loudly
when its CUDA library is missing.

It is an FP64 numpy restatement of the reference's algorithm:

* ``se3``        -- jaxlie-convention SE(3) (wxyz_xyz, tangent [v, w]).
* ``kinematics`` -- full config (mimic/fixed), FK over a topologically
  sorted joint tree, link-pose gather, FK depth schedule, ancestor masks.
* ``collision``  -- signed-distance primitives (CUDA and JAX conventions),
  sphere transforms, world / self reductions, hinge-squared costs.
* ``lm``         -- multi-seed Levenberg-Marquardt IK step for step as the
  reference CUDA kernel, vectorised over seeds; FP64 pose errors.
* ``traj``       -- CHOMP trajectory cost (smoothness + limits + collision
  hinge) and its gradient by central finite differences.

Parity status: the reference's own JAX path (jax/jaxlie) is not installed
in this image, so the oracle is pinned against the reference's CUDA helper
functions compiled for the host from their own sources (``oracle/_ref``,
recipe ``oracle/Makefile``), through the golden vectors committed in
``tests/golden/`` (script ``tests/golden/make_golden.py``).  The LM loop
itself has no reference-produced golden vector; it is pinned only through
its pinned components (FK, residual, Jacobian, Cholesky, distances).
"""
