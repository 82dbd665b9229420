"""FP64 signed distances and collision reductions -- oracle (test infrastructure only).

Conventions (positive = separated, negative = penetration):

* CUDA convention, ``src/pyroffi/cuda_kernels/_collision_cuda_helpers.cuh:14-175``
  (sphere-sphere, sphere-capsule with the 1e-12 degenerate-segment guard,
  box SDF in the box frame spanned by the three stored axis columns,
  halfspace, capsule pairs, ``colldist_from_sdf``);
* JAX convention, ``src/pyroffi/collision/_geometry_pairs.py:13-275`` with
  ``_utils.normalize_with_norm`` (norm of ``x + 1e-6``, ``_utils.py:41-50``) and
  the ``+1e-12`` inside the box SDF square root (``_geometry_pairs.py:268``).

World obstacle arrays follow ``_extract_world_arrays``
(``src/pyroffi/collision/_cuda_collision.py:98-168``): spheres ``[Ms,4]``
(x,y,z,r), capsules ``[Mc,7]`` (p1, p2, r), boxes ``[Mb,15]`` (centre, axis
columns a1,a2,a3, half-lengths), halfspaces ``[Mh,6]`` (normal, point).  The
obstacle axis of every ``[.., M]`` output is spheres, capsules, boxes,
halfspaces in that order.

Reductions:

* ``world_sphere``          -- ``wcs_vs_*`` (``_collision_cuda_kernel.cu:64-165``):
  ``[B,K,M]``, padding spheres (radius < 0) give 1e9;
* ``world_sphere_reduced``  -- ``wcsr_vs_*`` (``:170-304``): ``[B,N,M]`` min over
  s with sphere k = s*N + n, padding skipped, 1e9 when a link has none;
* ``self_sphere_full``      -- ``self_collision_sphere_kernel`` (``:426-470``):
  min over all S x S sphere pairs of the two links;
* ``self_sphere_diag``      -- ``compute_self_collision_distance``
  (``src/pyroffi/collision/_robot_collision.py:796-828``): min over s of the
  distance between sphere s of link i and sphere s of link j;
* ``lm_penalty``            -- the LS-IK hinge penalty
  (``src/pyroffi/cuda_kernels/_ls_ik_cuda_kernel.cu:166-229``);
* ``chomp_collision_cost``  -- ``_collision_cost``
  (``src/pyroffi/optimization_engines/_chomp_optimization.py:124-153``).
"""

from __future__ import annotations

import numpy as np

from . import se3

BIG = 1e9


# ---------------------------------------------------------------------------
# primitives, CUDA convention
# ---------------------------------------------------------------------------

def sphere_sphere(a, ar, b, br):
    return np.linalg.norm(np.asarray(a) - np.asarray(b), axis=-1) - (ar + br)


def sphere_capsule(s, sr, p1, p2, cr):
    v = p2 - p1
    len2 = np.sum(v * v, axis=-1)
    t = np.where(len2 > 1e-12, np.sum((s - p1) * v, axis=-1) / np.where(len2 > 1e-12, len2, 1.0), 0.0)
    t = np.clip(t, 0.0, 1.0)
    c = p1 + t[..., None] * v
    return np.linalg.norm(s - c, axis=-1) - (sr + cr)


def box_sdf_local(p, hl):
    q = np.abs(p) - hl
    return np.linalg.norm(np.maximum(q, 0.0), axis=-1) + np.minimum(np.max(q, axis=-1), 0.0)


def sphere_box(s, sr, box):
    d = s - box[..., 0:3]
    local = np.stack([np.sum(d * box[..., 3:6], -1), np.sum(d * box[..., 6:9], -1),
                      np.sum(d * box[..., 9:12], -1)], axis=-1)
    return box_sdf_local(local, box[..., 12:15]) - sr


def sphere_halfspace(s, sr, hs):
    return np.sum((s - hs[..., 3:6]) * hs[..., 0:3], axis=-1) - sr


def capsule_capsule(a1, a2, ar, b1, b2, br):
    """Closest points between segments (clamped), as the CUDA helper."""
    d1 = a2 - a1
    d2 = b2 - b1
    r = a1 - b1
    a = np.sum(d1 * d1, -1)
    e = np.sum(d2 * d2, -1)
    f = np.sum(d2 * r, -1)
    c = np.sum(d1 * r, -1)
    b = np.sum(d1 * d2, -1)
    eps = 1e-10
    a, e, f, c, b = np.broadcast_arrays(a, e, f, c, b)
    s = np.zeros(a.shape)
    t = np.zeros(a.shape)
    for idx in np.ndindex(a.shape):
        ai, ei, fi, ci, bi = a[idx], e[idx], f[idx], c[idx], b[idx]
        if ai <= eps and ei <= eps:
            si = ti = 0.0
        elif ai <= eps:
            si = 0.0
            ti = min(max(fi / ei, 0.0), 1.0)
        elif ei <= eps:
            ti = 0.0
            si = min(max(-ci / ai, 0.0), 1.0)
        else:
            den = ai * ei - bi * bi
            si = min(max((bi * fi - ci * ei) / den, 0.0), 1.0) if abs(den) > eps else 0.0
            ti = (bi * si + fi) / ei
            if ti < 0.0:
                ti = 0.0
                si = min(max(-ci / ai, 0.0), 1.0)
            elif ti > 1.0:
                ti = 1.0
                si = min(max((bi - ci) / ai, 0.0), 1.0)
        s[idx], t[idx] = si, ti
    p = a1 + s[..., None] * d1 - (b1 + t[..., None] * d2)
    return np.linalg.norm(p, axis=-1) - (ar + br)


def capsule_box(p1, p2, cr, box):
    c = box[..., 0:3]
    ax = [box[..., 3:6], box[..., 6:9], box[..., 9:12]]
    al = np.stack([np.sum((p1 - c) * a, -1) for a in ax], -1)
    bl = np.stack([np.sum((p2 - c) * a, -1) for a in ax], -1)
    ab = bl - al
    l2 = np.sum(ab * ab, -1)
    t = np.where(l2 > 1e-12, np.sum(-al * ab, -1) / np.where(l2 > 1e-12, l2, 1.0), 0.0)
    t = np.clip(t, 0.0, 1.0)
    return box_sdf_local(al + t[..., None] * ab, box[..., 12:15]) - cr


def capsule_halfspace(p1, p2, cr, hs):
    d1 = np.sum((p1 - hs[..., 3:6]) * hs[..., 0:3], -1)
    d2 = np.sum((p2 - hs[..., 3:6]) * hs[..., 0:3], -1)
    return np.minimum(d1, d2) - cr


def colldist_from_sdf(d, margin):
    d = np.minimum(d, margin)
    val = np.where(d < 0.0, d - 0.5 * margin, -0.5 / (margin + 1e-6) * (d - margin) ** 2)
    return np.minimum(val, 0.0)


# ---------------------------------------------------------------------------
# primitives, JAX convention (for documenting the +1e-6 bias)
# ---------------------------------------------------------------------------

def jax_sphere_sphere(a, ar, b, br):
    return np.linalg.norm((np.asarray(b) - np.asarray(a)) + 1e-6, axis=-1) - (ar + br)


def jax_box_sphere(s, sr, box):
    d = s - box[..., 0:3]
    local = np.stack([np.sum(d * box[..., 3:6], -1), np.sum(d * box[..., 6:9], -1),
                      np.sum(d * box[..., 9:12], -1)], axis=-1)
    q = np.abs(local) - box[..., 12:15]
    outside = np.sqrt(np.sum(np.maximum(q, 0.0) ** 2, -1) + 1e-12)
    return outside + np.minimum(np.max(q, -1), 0.0) - sr


# ---------------------------------------------------------------------------
# robot-level
# ---------------------------------------------------------------------------

def transform_points(T, p):
    """Apply poses T [..., 7] to points p [..., 3] (broadcasting)."""
    return se3.apply(T, p)


def point_vs_world(p, r, ws, wc, wb, wh):
    """Distances [..., M] from spheres (p [...,3], r [...]) to all obstacles."""
    p = np.asarray(p, np.float64)
    r = np.asarray(r, np.float64)
    parts = []
    pe = p[..., None, :]
    re = r[..., None]
    if len(ws):
        parts.append(sphere_sphere(pe, re, ws[:, :3], ws[:, 3]))
    if len(wc):
        parts.append(sphere_capsule(pe, re, wc[:, 0:3], wc[:, 3:6], wc[:, 6]))
    if len(wb):
        parts.append(sphere_box(pe, re, np.asarray(wb, np.float64)))
    if len(wh):
        parts.append(sphere_halfspace(pe, re, np.asarray(wh, np.float64)))
    if not parts:
        return np.zeros((*p.shape[:-1], 0))
    return np.concatenate(parts, axis=-1)


def world_sphere(centers_bk3, radii_bk, ws, wc, wb, wh):
    """[B,K,M] per-sphere distances; padding (radius < 0) rows are 1e9."""
    d = point_vs_world(centers_bk3, radii_bk, ws, wc, wb, wh)
    return np.where(np.asarray(radii_bk)[..., None] < 0, BIG, d)


def world_sphere_reduced(centers_bk3, radii_bk, ws, wc, wb, wh, n):
    """[B,N,M]: min over s of sphere k = s*N + n, skipping padding."""
    B, K, _ = centers_bk3.shape
    S = K // n
    d = point_vs_world(centers_bk3, radii_bk, ws, wc, wb, wh)        # [B,K,M]
    d = np.where(np.asarray(radii_bk)[..., None] < 0, np.inf, d)
    d = d[:, : S * n].reshape(B, S, n, d.shape[-1]).min(axis=1)
    return np.where(np.isinf(d), BIG, d)


def self_sphere_full(centers_bsn3, radii_bsn, pair_i, pair_j):
    """[B,P]: min over all sphere pairs (si of link i, sj of link j)."""
    ci = centers_bsn3[:, :, pair_i, :]                 # [B,S,P,3]
    cj = centers_bsn3[:, :, pair_j, :]
    ri = radii_bsn[:, :, pair_i]
    rj = radii_bsn[:, :, pair_j]
    d = sphere_sphere(ci[:, :, None], ri[:, :, None], cj[:, None, :], rj[:, None, :])  # [B,S,S,P]
    valid = (ri[:, :, None] >= 0) & (rj[:, None, :] >= 0)
    d = np.where(valid, d, BIG)
    return np.minimum(d.min(axis=(1, 2)), BIG)


def self_sphere_diag(centers_bsn3, radii_bsn, pair_i, pair_j):
    """[B,P]: min over s of d(sphere (i,s), sphere (j,s)) (padding -> huge)."""
    ci = centers_bsn3[:, :, pair_i, :]
    cj = centers_bsn3[:, :, pair_j, :]
    d = sphere_sphere(ci, radii_bsn[:, :, pair_i], cj, radii_bsn[:, :, pair_j])
    return d.min(axis=1)


def robot_sphere_world(T_joints, spheres_local, sphere_joint):
    """World centres [..., n_rs, 3] of spheres given in their joint frames."""
    T = T_joints[..., np.asarray(sphere_joint), :]
    return se3.apply(T, np.asarray(spheres_local, np.float64)[:, :3])


def lm_penalty(T_joints, spheres_local, sphere_joint, ws, wc, wb, wh, margin,
               weight, self_i=None, self_j=None):
    """LS-IK hinge penalty: weight * sum over (robot sphere, obstacle) with
    d < margin of (d - margin)^2, plus the same over explicit robot-sphere
    pairs (self_i, self_j) when given."""
    sj = np.asarray(sphere_joint)
    valid = (sj >= 0) & (sj < T_joints.shape[-2])
    p = robot_sphere_world(T_joints, np.asarray(spheres_local)[valid], sj[valid])
    r = np.asarray(spheres_local, np.float64)[valid, 3]
    d = point_vs_world(p, r, ws, wc, wb, wh)
    pen = np.sum(np.where(d < margin, (d - margin) ** 2, 0.0), axis=(-1, -2))
    if self_i is not None and len(self_i):
        P_all = robot_sphere_world(T_joints, spheres_local, np.where(valid, sj, 0))
        r_all = np.asarray(spheres_local, np.float64)[:, 3]
        ds = sphere_sphere(P_all[..., self_i, :], r_all[self_i], P_all[..., self_j, :], r_all[self_j])
        pen = pen + np.sum(np.where(ds < margin, (ds - margin) ** 2, 0.0), axis=-1)
    return weight * pen


def chomp_collision_cost(link_T, centers_local_ns3, radii_ns, pair_i, pair_j,
                         ws, wc, wb, wh, margin):
    """Per-configuration CHOMP collision cost: sum over self pairs (diag-S)
    and world [N,M] (min over S) of max(0, margin - d)^2.

    link_T [..., N, 7]; centers_local_ns3 [N,S,3] in link frames; radii_ns [N,S].
    """
    c = se3.apply(link_T[..., :, None, :], centers_local_ns3)          # [...,N,S,3]
    r = np.broadcast_to(radii_ns, c.shape[:-1])
    lead = c.shape[:-3]
    cf = c.reshape(-1, *c.shape[-3:])
    rf = r.reshape(-1, *r.shape[-2:])
    # self: [B,S,N,3] ordering
    cs = np.swapaxes(cf, 1, 2)
    rs = np.swapaxes(rf, 1, 2)
    total = np.zeros(cf.shape[0])
    if len(pair_i):
        dself = self_sphere_diag(cs, rs, np.asarray(pair_i), np.asarray(pair_j))
        total += np.sum(np.maximum(0.0, margin - dself) ** 2, axis=-1)
    dw = point_vs_world(cf, rf, ws, wc, wb, wh)                       # [B,N,S,M]
    dmin = dw.min(axis=2)                                              # [B,N,M]
    total += np.sum(np.maximum(0.0, margin - dmin) ** 2, axis=(-1, -2))
    return total.reshape(lead)
