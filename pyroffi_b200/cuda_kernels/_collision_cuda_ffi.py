"""Collision-distance drop-ins for ``src/pyroffi/cuda_kernels/_collision_cuda_ffi.py:70-242``.

Same names, argument order, layouts and outputs (torch CUDA tensors):

* ``collision_world_sphere(centers[3,B,K], radii[B,K], ws, wc, wb, wh) -> [B,K,M]``
* ``collision_world_sphere_reduced(..., n) -> [B,N,M]``
* ``collision_world_capsule(caps[7,B,N], ws, wc, wb, wh) -> [B,N,M]``
* ``collision_self_sphere(centers[B,S,N,3], radii[B,S,N], pair_i, pair_j) -> [B,P]``
* ``collision_self_capsule(caps[B,N,7], pair_i, pair_j) -> [B,P]``

with M = Ms + Mc + Mb + Mh (spheres, capsules, boxes, halfspaces) and the
empty-world / empty-pair shortcuts of the reference.
"""

from __future__ import annotations

import torch

from .. import _lib
from .._tensors import f32, i32, ptr, require_cuda, stream_ptr


def _world(dev, ws, wc, wb, wh):
    w = [f32(x).to(dev) for x in (ws, wc, wb, wh)]
    return w, [int(x.shape[0]) for x in w]


def collision_world_sphere(sphere_centers, sphere_radii, world_spheres, world_capsules,
                           world_boxes, world_halfspaces) -> torch.Tensor:
    dev = require_cuda(sphere_centers)
    B, K = int(sphere_centers.shape[1]), int(sphere_centers.shape[2])
    w, (Ms, Mc, Mb, Mh) = _world(dev, world_spheres, world_capsules, world_boxes, world_halfspaces)
    M = Ms + Mc + Mb + Mh
    out = torch.empty((B, K, M), dtype=torch.float32, device=dev)
    if M == 0:
        return out
    c, r = f32(sphere_centers), f32(sphere_radii).to(dev)
    _lib.call("pk_collision_world_sphere", stream_ptr(dev), ptr(c), ptr(r), *[ptr(x) for x in w],
              ptr(out), B, K, Ms, Mc, Mb, Mh)
    return out


def collision_world_sphere_reduced(sphere_centers, sphere_radii, world_spheres, world_capsules,
                                   world_boxes, world_halfspaces, n: int) -> torch.Tensor:
    dev = require_cuda(sphere_centers)
    B, K = int(sphere_centers.shape[1]), int(sphere_centers.shape[2])
    w, (Ms, Mc, Mb, Mh) = _world(dev, world_spheres, world_capsules, world_boxes, world_halfspaces)
    M = Ms + Mc + Mb + Mh
    out = torch.empty((B, int(n), M), dtype=torch.float32, device=dev)
    if M == 0:
        return out
    c, r = f32(sphere_centers), f32(sphere_radii).to(dev)
    _lib.call("pk_collision_world_sphere_reduced", stream_ptr(dev), ptr(c), ptr(r),
              *[ptr(x) for x in w], ptr(out), B, K, Ms, Mc, Mb, Mh, int(n))
    return out


def collision_world_capsule(caps, world_spheres, world_capsules, world_boxes,
                            world_halfspaces) -> torch.Tensor:
    dev = require_cuda(caps)
    B, N = int(caps.shape[1]), int(caps.shape[2])
    w, (Ms, Mc, Mb, Mh) = _world(dev, world_spheres, world_capsules, world_boxes, world_halfspaces)
    M = Ms + Mc + Mb + Mh
    out = torch.empty((B, N, M), dtype=torch.float32, device=dev)
    if M == 0:
        return out
    c = f32(caps)
    _lib.call("pk_collision_world_capsule", stream_ptr(dev), ptr(c), *[ptr(x) for x in w], ptr(out),
              B, N, Ms, Mc, Mb, Mh)
    return out


def collision_self_sphere(sphere_centers, sphere_radii, pair_i, pair_j) -> torch.Tensor:
    dev = require_cuda(sphere_centers)
    B, S, N = (int(x) for x in sphere_centers.shape[:3])
    P = int(pair_i.shape[0])
    out = torch.empty((B, P), dtype=torch.float32, device=dev)
    if P == 0:
        return out
    c, r = f32(sphere_centers), f32(sphere_radii).to(dev)
    pi, pj = i32(pair_i).to(dev), i32(pair_j).to(dev)
    _lib.call("pk_collision_self_sphere", stream_ptr(dev), ptr(c), ptr(r), ptr(pi), ptr(pj), ptr(out),
              B, S, N, P)
    return out


def collision_self_capsule(caps, pair_i, pair_j) -> torch.Tensor:
    dev = require_cuda(caps)
    B, N = int(caps.shape[0]), int(caps.shape[1])
    P = int(pair_i.shape[0])
    out = torch.empty((B, P), dtype=torch.float32, device=dev)
    if P == 0:
        return out
    c = f32(caps)
    pi, pj = i32(pair_i).to(dev), i32(pair_j).to(dev)
    _lib.call("pk_collision_self_capsule", stream_ptr(dev), ptr(c), ptr(pi), ptr(pj), ptr(out), B, N, P)
    return out
