"""pyroffi_b200 -- B200-native (sm_100a) kinematics hot path of pyroffi.

Batched FK over SE(3) joint trees, collision-sphere world transforms,
sphere / capsule / box / halfspace signed distances and self distances,
multi-seed Levenberg-Marquardt IK with a collision penalty and FP64
re-verification, all as hand-written CUDA kernels behind the C-ABI in
``include/pyroffi_b200.h``.  There is no CPU fallback.
"""

from . import robot, workloads  # noqa: F401
from .urdf import load_urdf  # noqa: F401

__version__ = "0.1.0"
