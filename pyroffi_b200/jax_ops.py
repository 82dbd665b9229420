"""The trajectory cost behind ``jax.custom_vjp`` (needs jax; import-guarded).

The reference differentiates CHOMP's cost with ``jax.value_and_grad``
(``src/pyroffi/optimization_engines/_chomp_optimization.py:243-263``).  Here
the same cost has a hand-written adjoint kernel (``pk_traj_cost_grad``), and
this module puts it behind ``jax.custom_vjp`` exactly as
``pyroffi_b200.trajopt.TrajectoryCostFn`` puts it behind
``torch.autograd.Function``:

* ``fwd`` runs the kernel for the cost only (``grad = NULL``) and keeps the
  trajectory as the residual -- no link transform is stored;
* ``bwd`` runs it again for the gradient only (``cost = NULL``), recomputing
  the link transforms, and scales row ``b`` by the cotangent ``ct[b]``.

Arrays cross between jax and torch by DLPack, so the device buffers are
shared, not copied, and the kernel runs on torch's current stream of that
device (the function synchronises nothing).  This works on concrete jax
arrays on a CUDA device.  Under ``jax.jit`` the inputs are tracers with no
buffer behind them: there the kernel has to be an XLA custom call, i.e. the
XLA FFI handler over ``pk_traj_cost_grad`` that the integration notes
describe, and calling this function on a tracer raises a ``TypeError`` that
says so.

    import jax.numpy as jnp
    from pyroffi_b200.trajopt import TrajectoryCost
    from pyroffi_b200.jax_ops import traj_cost_vjp

    cost = traj_cost_vjp(TrajectoryCost(model, spheres, world, pairs))
    J, vjp = jax.vjp(cost, traj)            # traj: jax array [B, T, n] on a GPU
    (g,) = vjp(jnp.ones_like(J))            # == dJ/dtraj from the adjoint kernel
"""

from __future__ import annotations

try:  # jax is optional: the rest of the package never needs it
    import jax
    import jax.dlpack as _jdl
except ImportError as _e:  # pragma: no cover - depends on the environment
    jax = None
    _IMPORT_ERROR = _e
else:
    _IMPORT_ERROR = None

import torch

from .trajopt import TrajectoryCost


def _require_jax():
    if jax is None:
        raise ImportError("pyroffi_b200.jax_ops needs jax; it is not installed") from _IMPORT_ERROR


def _to_torch(x) -> torch.Tensor:
    if isinstance(x, jax.core.Tracer):
        raise TypeError("traj_cost_vjp runs on concrete jax arrays; under jax.jit register the XLA FFI handler "
                        "over pk_traj_cost_grad and call it with jax.ffi.ffi_call instead")
    return torch.from_dlpack(x)


def _to_jax(t: torch.Tensor):
    return _jdl.from_dlpack(t.contiguous())


def traj_cost_vjp(cost_obj: TrajectoryCost):
    """J = f(traj) with traj [B, T, n] f32 (a jax array on the cost's CUDA
    device) and J [B]; ``jax.vjp`` / ``jax.grad`` of ``f`` use the adjoint kernel."""
    _require_jax()

    @jax.custom_vjp
    def f(traj):
        return _to_jax(cost_obj.cost(_to_torch(traj)))

    def fwd(traj):
        return f(traj), traj

    def bwd(traj, ct):
        g = cost_obj.grad(_to_torch(traj))
        c = _to_torch(ct).to(device=g.device, dtype=g.dtype)
        return (_to_jax(c[:, None, None] * g),)

    f.defvjp(fwd, bwd)
    return f
