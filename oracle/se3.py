"""FP64 SE(3) in the jaxlie convention -- oracle (test infrastructure only).

Storage is ``wxyz_xyz``: a unit quaternion (w, x, y, z) followed by a
translation (tx, ty, tz).  Tangents are ``[v, omega]`` (linear first), as
in jaxlie 1.5.0, which the reference uses for ``SE3.exp`` / ``@`` /
``inverse().log()`` (``src/pyroffi/_robot.py:212-216``,
``src/pyroffi/optimization_engines/_ik_primitives.py:103``) and restates in
``src/pyroffi/cuda_kernels/_fk_cuda_helpers.cuh:29-133``.

jaxlie itself is a third-party dependency absent from the reference tree
(pinned ``jaxlie==1.5.0`` in ``pyproject.toml``); these are the published
formulas (exponential map with A = sin t / t, B = (1 - cos t)/t^2,
C = (t - sin t)/t^3; logarithm with the inverse of V), written for numpy
and vectorised over any leading batch shape.  Small angles use Taylor series
so FP64 stays accurate at theta -> 0.
"""

from __future__ import annotations

import numpy as np


def identity(shape=()) -> np.ndarray:
    T = np.zeros((*shape, 7), dtype=np.float64)
    T[..., 0] = 1.0
    return T


def quat_mul(q1: np.ndarray, q2: np.ndarray) -> np.ndarray:
    """Hamilton product of wxyz quaternions (broadcasting)."""
    w1, x1, y1, z1 = np.moveaxis(q1, -1, 0)
    w2, x2, y2, z2 = np.moveaxis(q2, -1, 0)
    return np.stack(
        [
            w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2,
            w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
            w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
            w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2,
        ],
        axis=-1,
    )


def quat_conj(q: np.ndarray) -> np.ndarray:
    return q * np.array([1.0, -1.0, -1.0, -1.0])


def quat_rotate(q: np.ndarray, v: np.ndarray) -> np.ndarray:
    """Rotate 3-vectors ``v`` by unit quaternions ``q`` (v' = q v q*)."""
    w = q[..., :1]
    u = q[..., 1:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def quat_to_matrix(q: np.ndarray) -> np.ndarray:
    w, x, y, z = np.moveaxis(q, -1, 0)
    R = np.stack(
        [
            1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
            2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
            2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
        ],
        axis=-1,
    )
    return R.reshape(*R.shape[:-1], 3, 3)


def matrix_to_quat(R: np.ndarray) -> np.ndarray:
    """Rotation matrix -> unit wxyz quaternion with w >= 0 (Shepperd's method)."""
    R = np.asarray(R, dtype=np.float64)
    shp = R.shape[:-2]
    R = R.reshape(-1, 3, 3)
    q = np.empty((R.shape[0], 4))
    for i, m in enumerate(R):
        tr = m[0, 0] + m[1, 1] + m[2, 2]
        if tr > 0:
            s = 2.0 * np.sqrt(tr + 1.0)
            q[i] = [0.25 * s, (m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s]
        elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
            s = 2.0 * np.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2])
            q[i] = [(m[2, 1] - m[1, 2]) / s, 0.25 * s, (m[0, 1] + m[1, 0]) / s, (m[0, 2] + m[2, 0]) / s]
        elif m[1, 1] > m[2, 2]:
            s = 2.0 * np.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2])
            q[i] = [(m[0, 2] - m[2, 0]) / s, (m[0, 1] + m[1, 0]) / s, 0.25 * s, (m[1, 2] + m[2, 1]) / s]
        else:
            s = 2.0 * np.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1])
            q[i] = [(m[1, 0] - m[0, 1]) / s, (m[0, 2] + m[2, 0]) / s, (m[1, 2] + m[2, 1]) / s, 0.25 * s]
        if q[i, 0] < 0:
            q[i] = -q[i]
        q[i] /= np.linalg.norm(q[i])
    return q.reshape(*shp, 4)


def compose(T1: np.ndarray, T2: np.ndarray) -> np.ndarray:
    """T1 @ T2 (jaxlie ``SE3.__matmul__``)."""
    q = quat_mul(T1[..., :4], T2[..., :4])
    t = quat_rotate(T1[..., :4], T2[..., 4:7]) + T1[..., 4:7]
    return np.concatenate([q, t], axis=-1)


def inverse(T: np.ndarray) -> np.ndarray:
    qi = quat_conj(T[..., :4])
    return np.concatenate([qi, -quat_rotate(qi, T[..., 4:7])], axis=-1)


def apply(T: np.ndarray, p: np.ndarray) -> np.ndarray:
    return quat_rotate(T[..., :4], p) + T[..., 4:7]


def _skew_apply(w: np.ndarray, v: np.ndarray) -> np.ndarray:
    return np.cross(w, v)


def exp(tangent: np.ndarray) -> np.ndarray:
    """SE(3) exponential of ``[v, omega]`` tangents (jaxlie ``SE3.exp``)."""
    tangent = np.asarray(tangent, dtype=np.float64)
    v = tangent[..., :3]
    w = tangent[..., 3:6]
    th2 = np.sum(w * w, axis=-1)
    small = th2 < 1e-8
    th2s = np.where(small, 1.0, th2)
    th = np.sqrt(th2s)
    half = 0.5 * th
    # rotation
    s_half_over_th = np.where(small, 0.5 - th2 / 48.0 + th2 * th2 / 3840.0, np.sin(half) / th)
    qw = np.where(small, 1.0 - th2 / 8.0 + th2 * th2 / 384.0, np.cos(half))
    q = np.concatenate([qw[..., None], s_half_over_th[..., None] * w], axis=-1)
    # V = I + B [w]x + C [w]x^2
    B = np.where(small, 0.5 - th2 / 24.0 + th2 * th2 / 720.0, (1.0 - np.cos(th)) / th2s)
    C = np.where(small, 1.0 / 6.0 - th2 / 120.0 + th2 * th2 / 5040.0, (th - np.sin(th)) / (th2s * th))
    wxv = _skew_apply(w, v)
    wxwxv = _skew_apply(w, wxv)
    t = v + B[..., None] * wxv + C[..., None] * wxwxv
    return np.concatenate([q, t], axis=-1)


def so3_log(q: np.ndarray) -> np.ndarray:
    """SO(3) logarithm of wxyz quaternions (shortest rotation vector)."""
    q = np.asarray(q, dtype=np.float64)
    w = q[..., 0]
    u = q[..., 1:4]
    n2 = np.sum(u * u, axis=-1)
    n = np.sqrt(n2)
    small = n2 < 1e-16
    ws = np.where(w == 0.0, 1e-300, w)
    # 2 * atan2(n, |w|) / n with the sign of w folded into the factor.
    big_factor = 2.0 * np.arctan2(np.where(w < 0, -n, n), np.abs(w)) / np.where(small, 1.0, n)
    taylor = 2.0 / ws - 2.0 / 3.0 * n2 / (ws ** 3)
    factor = np.where(small, taylor, big_factor)
    return factor[..., None] * u


def log(T: np.ndarray) -> np.ndarray:
    """SE(3) logarithm -> ``[v, omega]`` (jaxlie ``SE3.log``)."""
    w = so3_log(T[..., :4])
    t = T[..., 4:7]
    th2 = np.sum(w * w, axis=-1)
    small = th2 < 1e-8
    th2s = np.where(small, 1.0, th2)
    th = np.sqrt(th2s)
    half = 0.5 * th
    # V^{-1} = I - 1/2 [w]x + (1 - (th/2) cot(th/2)) / th^2 [w]x^2
    coef = np.where(small, 1.0 / 12.0 + th2 / 720.0, (1.0 - half * np.cos(half) / np.sin(half)) / th2s)
    wxt = np.cross(w, t)
    v = t - 0.5 * wxt + coef[..., None] * np.cross(w, wxt)
    return np.concatenate([v, w], axis=-1)


def rotation_angle(q: np.ndarray) -> np.ndarray:
    """Angle of the rotation ``q`` in [0, pi]: ||SO3.log(q)||."""
    return np.linalg.norm(so3_log(q), axis=-1)


def random_unit_quat(rng: np.random.Generator, shape=()) -> np.ndarray:
    q = rng.normal(size=(*shape, 4))
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    return np.where(q[..., :1] < 0, -q, q)
