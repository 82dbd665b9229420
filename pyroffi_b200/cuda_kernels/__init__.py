"""Drop-in operators with the reference's ``src/pyroffi/cuda_kernels`` names and
argument meaning, on torch CUDA tensors, calling the sm_100a C-ABI."""

from ._fk_cuda import fk_cuda
from ._collision_cuda_ffi import (
    collision_self_capsule,
    collision_self_sphere,
    collision_world_capsule,
    collision_world_sphere,
    collision_world_sphere_reduced,
)
from ._ls_ik_cuda import ls_ik_cuda

__all__ = [
    "fk_cuda",
    "collision_world_sphere",
    "collision_world_sphere_reduced",
    "collision_world_capsule",
    "collision_self_sphere",
    "collision_self_capsule",
    "ls_ik_cuda",
]
