"""ctypes binding of the oracle's C port (``oracle/cpu/pk_cpu.c``) -- TEST
AND BASELINE INFRASTRUCTURE ONLY.

The C port restates the reference LM kernel (``ls_ik_lm_kernel``,
``src/pyroffi/cuda_kernels/_ls_ik_cuda_kernel.cu:65-394``) per seed in FP32
with FP64 normal equations, OpenMP over seeds.  The tests use it as the
full-size parity reference of the IK workload, and ``bench.py`` times it as
the CPU baseline; nothing in ``pyroffi_b200`` loads it.
"""

from __future__ import annotations

import ctypes as C
import subprocess
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SO = HERE / "_build" / "libpk_cpu.so"


def load() -> C.CDLL:
    if not SO.exists():
        subprocess.run(["make", "-C", str(HERE), "cpu"], check=True, capture_output=True)
    lib = C.CDLL(str(SO))
    lib.pk_cpu_max_threads.restype = C.c_int
    return lib


def max_threads(lib) -> int:
    return int(lib.pk_cpu_max_threads())


def ls_ik(lib, w, p0: int, n_prob: int, n_threads: int):
    """The port on problems [p0, p0 + n_prob) of an IK workload (``workloads.ik``):
    returns (seconds, cfgs [n_prob, Sd, n], errs [n_prob, Sd])."""
    m = w.model
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)

    f32, i32 = np.float32, np.int32
    seeds = np.ascontiguousarray(w.seeds[p0:p0 + n_prob], f32)
    tgt = np.ascontiguousarray(w.target_T[p0:p0 + n_prob, None, :], f32)
    out_cfg = np.zeros_like(seeds)
    out_err = np.zeros(seeds.shape[:2], f32)
    tj = np.asarray([m.link_joint(w.target_link)], i32)
    anc = m.ancestor_mask(w.target_link)[None]
    fp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    t0 = time.perf_counter()
    st = lib.pk_cpu_ls_ik(
        fp(seeds), arr(m.twists, f32), arr(m.parent_tf, f32), arr(m.parent_idx, i32), arr(m.act_idx, i32),
        arr(m.mimic_mul, f32), arr(m.mimic_off, f32), arr(m.mimic_act_idx, i32), arr(m.topo_inv, i32),
        arr(tj, i32), arr(anc, i32), fp(tgt), arr(w.spheres_local, f32), arr(w.sphere_joint, i32),
        arr(w.world.spheres, f32), arr(w.self_pairs[:, 0], i32), arr(w.self_pairs[:, 1], i32),
        arr(m.lower, f32), arr(m.upper, f32), arr(np.zeros(m.n_act), i32), fp(out_cfg), fp(out_err),
        C.c_int(n_prob), C.c_int(seeds.shape[1]), C.c_int(m.n_act), C.c_int(m.n_joints), C.c_int(1),
        C.c_int(len(w.spheres_local)), C.c_int(len(w.world.spheres)), C.c_int(len(w.self_pairs)),
        C.c_int(w.max_iter), C.c_float(w.pos_weight), C.c_float(w.ori_weight), C.c_float(w.lambda_init),
        C.c_float(w.lambda_down), C.c_float(w.lambda_up), C.c_float(1e-8), C.c_float(1e-8), C.c_int(1),
        C.c_float(w.collision_weight), C.c_float(w.collision_margin), C.c_int(n_threads))
    dt = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError(f"pk_cpu_ls_ik failed ({st})")
    return dt, out_cfg, out_err


def success(w, p0: int, cfgs, errs):
    """Per-problem FP64 success (1 mm / 0.01 rad) of the winners of (cfgs, errs),
    problems [p0, p0 + len(cfgs)) of the workload."""
    from . import lm as olm

    win, _ = olm.select_winner(np.asarray(cfgs, np.float64), errs)
    pe, re = olm.pose_errors(win, w.target_T[p0:p0 + len(cfgs)].astype(np.float64), w.model.as_dict(),
                             w.model.link_joint(w.target_link))
    return (pe < w.pos_tol) & (re < w.rot_tol)
