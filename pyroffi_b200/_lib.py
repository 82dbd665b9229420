"""ctypes binding of ``libpyroffi_b200.so`` (the C-ABI in ``include/pyroffi_b200.h``).

The library is built in-tree (``python -m pyroffi_b200.build``).  There is
no fallback: if the library is missing or fails to load, every entry point
raises.  Status codes other than ``PK_OK`` raise :class:`PkError` with the
library's message.
"""

from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpyroffi_b200.so"

PK_OK, PK_ERR_INVALID, PK_ERR_CAPACITY, PK_ERR_CUDA, PK_ERR_TIMEOUT = 0, 1, 2, 3, 4

_p = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_f32 = C.c_float


class PkError(RuntimeError):
    def __init__(self, status: int, fn: str, msg: str):
        super().__init__(f"{fn} failed ({status}): {msg}")
        self.status = status


class LmOptions(C.Structure):
    """``pk_lm_options`` of the C-ABI."""

    _fields_ = [
        ("max_iter", _i32),
        ("pos_weight", _f32),
        ("ori_weight", _f32),
        ("lambda_init", _f32),
        ("lambda_down", _f32),
        ("lambda_up", _f32),
        ("eps_pos", _f32),
        ("eps_ori", _f32),
        ("enable_collision", _i32),
        ("collision_weight", _f32),
        ("collision_margin", _f32),
        ("threads_per_seed", _i32),
        ("seeds_per_block", _i32),
        ("lanes_per_wide_seed", _i32),
        ("fp64_solve", _i32),
        ("obstacle_grid", _i32),
    ]


# name -> argument types (after which the return type is int)
SIGNATURES: dict[str, list] = {
    "pk_fk_cuda": [_p] * 13 + [_i64, _i32, _i32, _i32],
    "pk_collision_world_sphere": [_p] * 8 + [_i64, _i32, _i32, _i32, _i32, _i32],
    "pk_collision_world_sphere_reduced": [_p] * 8 + [_i64, _i32, _i32, _i32, _i32, _i32, _i64],
    "pk_collision_world_capsule": [_p] * 7 + [_i64, _i32, _i32, _i32, _i32, _i32],
    "pk_collision_self_sphere": [_p] * 6 + [_i64, _i32, _i32, _i32],
    "pk_collision_self_capsule": [_p] * 5 + [_i64, _i32, _i32],
    "pk_ls_ik_cuda": [_p] * 22 + [_i64, _f32, _f32, _f32, _f32, _f32, _i64, _f32, _f32, _p, _p]
    + [_i32] * 10,
    "pk_ls_ik_ex": [_p, C.POINTER(LmOptions)] + [_p] * 25 + [_i32] * 11,
    "pk_ik_verify_select": [_p] * 4 + [_f32] + [_p] * 10 + [_f32, _f32] + [_p] * 4 + [_i32] * 5,
    "pk_fk_sphere_collision": [_p] * 21 + [_i64] + [_i32] * 8,
    "pk_ik_batch": [_p, C.POINTER(LmOptions), C.c_void_p, _i32] + [_p] * 4 + [_i32] * 4 + [_p, _i32, _p, _i32],
    "pk_ik_batch_static": [_p, C.POINTER(LmOptions), C.c_void_p, _i32] + [_p] * 4 + [_i32] * 4 + [_p, _i32, _i32],
    "pk_fp32_fma_peak": [_p, _p, _i32, _i32],
    "pk_traj_cost_grad": [_p, C.c_void_p] + [_p] * 22 + [_i64] + [_i32] * 10,
    "pk_hjcd_ik_coarse_cuda": [_p] + [_p] * 21 + [_i64, _i64, _f32, _f32, _p, _p] + [_i32] * 10,
    "pk_hjcd_ik_lm_cuda": [_p] + [_p] * 22 + [_i64, _i64, _f32, _f32, _f32, _f32, _f32, _i64, _f32, _f32, _p, _p,
                                              _p] + [_i32] * 10,
    "pk_sqp_ik_cuda": [_p] + [_p] * 21 + [_i64, _i64, _f32, _f32, _f32, _f32, _f32, _i64, _f32, _f32, _p, _p]
                      + [_i32] * 10,
    "pk_chomp_direction": [_p, _p, _p, _i64, _i32, _i32, _i32, _f32, _f32, _f32, _i32, _p],
    "pk_stage_wait_timeouts": [_p],
    "pk_stage_wait_reset": [],
    "pk_stage_wait_configure": [_i32, _i64],
    "pk_chomp_line_trials": [_p, _p, _p, _p, _i32, _f32, _p, _p, _p, _i64, _i32, _i32, _p],
    "pk_chomp_line_select": [_p, _p, _p, _p, _p, _p, _p, _i32, _f32, _i32, _i64, _i32, _i32],
    "pk_sco_linearize": [_p, C.c_void_p] + [_p] * 20 + [_i64] + [_i32] * 9,
    "pk_sco_inner": [_p, C.c_void_p] + [_p] * 8 + [_f32, _i64, _i32, _i32],
    "pk_sco_final_cost": [_p, C.c_void_p] + [_p] * 5 + [_i64, _i32, _i32],
    "pk_sco_workspace_bytes": [C.c_void_p, _i64, _i32, _i32, C.POINTER(C.c_size_t)],
    "pk_sco_trajopt": [_p, C.c_void_p] + [_p] * 24 + [C.c_size_t, _i64] + [_i32] * 10,
}


class IkClass(C.Structure):
    """``pk_ik_class`` of the C-ABI (one robot class of a batched IK call)."""

    _fields_ = [
        ("twists", _p), ("parent_tf", _p), ("parent_idx", _p), ("act_idx", _p), ("mimic_mul", _p),
        ("mimic_off", _p), ("mimic_act_idx", _p), ("topo_inv", _p), ("n_joints", _i32), ("n_act", _i32),
        ("target_jnts", _p), ("ancestor_masks", _p), ("target_Ts", _p), ("n_ee", _i32),
        ("robot_spheres_local", _p), ("robot_sphere_joint_idx", _p), ("n_robot_spheres", _i32),
        ("self_i", _p), ("self_j", _p), ("n_self", _i32),
        ("lower", _p), ("upper", _p), ("fixed_mask", _p),
        ("seeds", _p), ("out_cfg", _p), ("out_err", _p), ("n_problems", _i32), ("seed_stride", _i32),
        ("body", _i32),
    ]


class TrajOptions(C.Structure):
    """``pk_traj_options`` of the C-ABI."""

    _fields_ = [("margin", _f32), ("w_smooth", _f32), ("w_acc", _f32), ("w_jerk", _f32),
                ("w_limits", _f32), ("w_coll", _f32), ("active", C.c_void_p), ("active_period", _i64)]


class ScoOptions(C.Structure):
    """``pk_sco_options`` of the C-ABI."""

    _fields_ = [("n_outer_iters", _i32), ("n_inner_iters", _i32), ("m_lbfgs", _i32), ("w_smooth", _f32),
                ("w_acc", _f32), ("w_jerk", _f32), ("w_limits", _f32), ("w_trust", _f32), ("w_collision", _f32),
                ("w_collision_max", _f32), ("penalty_scale", _f32), ("collision_margin", _f32),
                ("smooth_min_temperature", _f32), ("fd_eps", _f32), ("self_all_pairs", _i32),
                ("inner_threads", _i32)]


_lock = threading.Lock()
_lib: C.CDLL | None = None


def load() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m pyroffi_b200.build` "
                "(there is no CPU fallback)")
        lib = C.CDLL(str(LIB_PATH))
        for name, argt in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argt
            fn.restype = C.c_int
        lib.pk_last_error.restype = C.c_char_p
        lib.pk_version.restype = C.c_char_p
        lib.pk_status_string.restype = C.c_char_p
        lib.pk_status_string.argtypes = [C.c_int]
        _lib = lib
        return lib


# PK_NVTX=1: every entry-point call is an NVTX range named after the entry
# point, so a timeline profiler shows the library's launches by name.
_NVTX = os.environ.get("PK_NVTX", "") not in ("", "0")


def call(name: str, *args) -> None:
    lib = load()
    if _NVTX:
        import torch

        torch.cuda.nvtx.range_push(name)
        try:
            st = getattr(lib, name)(*args)
        finally:
            torch.cuda.nvtx.range_pop()
    else:
        st = getattr(lib, name)(*args)
    if st != PK_OK:
        raise PkError(st, name, lib.pk_last_error().decode(errors="replace"))


def declared_symbols(header: Path | None = None) -> list[str]:
    """Function names declared in ``include/pyroffi_b200.h``."""
    import re

    header = header or Path(__file__).resolve().parent.parent / "include" / "pyroffi_b200.h"
    text = header.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(pk_\w+)\s*\(", text, re.M)))
