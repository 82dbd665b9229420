"""Tensor plumbing for the ctypes calls: dtype/contiguity coercion, pointers
and the current CUDA stream."""

from __future__ import annotations

import torch


def f32(t) -> torch.Tensor:
    t = torch.as_tensor(t)
    if t.dtype != torch.float32 or not t.is_contiguous():
        t = t.to(torch.float32).contiguous()
    return t


def i32(t) -> torch.Tensor:
    t = torch.as_tensor(t)
    if t.dtype != torch.int32 or not t.is_contiguous():
        t = t.to(torch.int32).contiguous()
    return t


def on_device(t: torch.Tensor, device: torch.device) -> torch.Tensor:
    if t.device != device:
        t = t.to(device)
    return t


def ptr(t: torch.Tensor | None) -> int | None:
    if t is None or t.numel() == 0:
        return None
    return t.data_ptr()


def stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(*ts: torch.Tensor) -> torch.device:
    dev = None
    for t in ts:
        if t is None:
            continue
        if not t.is_cuda:
            raise ValueError("pyroffi_b200 operators take CUDA tensors (there is no CPU path)")
        dev = t.device if dev is None else dev
        if t.device != dev:
            raise ValueError("all tensors must be on the same CUDA device")
    if dev is None:
        raise ValueError("no tensor given")
    return dev
