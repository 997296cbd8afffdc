"""Thin Python wrappers over the C-ABI kernels (device pointers from torch tensors).

Every wrapper launches on ``torch.cuda.current_stream()`` and returns without
synchronising unless it must read a result back.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib as L

_PARTIALS: dict = {}


def partials(device, n=L.PCG_PARTIALS) -> torch.Tensor:
    """A per-device float64 scratch for block partial sums (reused, never freed)."""
    key = (device, n)
    buf = _PARTIALS.get(key)
    if buf is None:
        buf = _PARTIALS[key] = torch.empty(n, dtype=torch.float64, device=device)
    return buf


def retract_group(entry, value: torch.Tensor, delta: torch.Tensor, lower=None, upper=None, delta_out=None):
    """X * Exp(delta) per variable of one group (float64 storage on the GPU).

    Known kinds run the CUDA retraction; a user-defined manifold (a Var with
    its own ``retract_fn`` and no CUDA kind) is retracted by ``vmap`` of its
    torch function on the device.
    """
    L.require_cuda(value, "retraction")
    kind = getattr(entry.var_type, "cuda_kind", None)
    if kind is None:
        return torch.func.vmap(entry.var_type.retract_fn)(value, delta.to(value.dtype))
    src = value if value.dtype == torch.float64 else value.double()
    src = src.contiguous()
    d = delta.to(torch.float64).contiguous()
    out = torch.empty_like(src)
    L.call("tls_retract", L.KIND[kind], entry.count, entry.dim, L.ptr(src), L.ptr(d), L.ptr(out), L.ptr(lower),
           L.ptr(upper), L.ptr(delta_out), L.stream_handle(value.device))
    return out if value.dtype == torch.float64 else out.to(value.dtype)


def reduce(x: torch.Tensor, op: int = 0) -> torch.Tensor:
    """Deterministic float64 sum (op 0), sum of squares (1) or abs-max (2) -> 0-dim tensor."""
    out = torch.empty((), dtype=torch.float64, device=x.device)
    if x.numel() == 0:
        return out.zero_()
    x = x.contiguous()
    L.call("tls_reduce", L.ptr(x), L.dtype_code(x.dtype), x.numel(), op, L.ptr(partials(x.device)), L.ptr(out),
           L.stream_handle(x.device))
    return out


def segment_reduce(seg: L.Segments, contrib: torch.Tensor, out: torch.Tensor, mode: int = 0, dim: int = 0):
    L.call("tls_segment_reduce", C.byref(seg), L.ptr(contrib), L.dtype_code(contrib.dtype), mode, dim, L.ptr(out),
           L.dtype_code(out.dtype), L.stream_handle(contrib.device))
    return out


def ordered_index_add_(out: torch.Tensor, index: torch.Tensor, source: torch.Tensor) -> torch.Tensor:
    """``out[index[k]] += source[k]`` with each target's contributions summed
    in ascending k by ``tls_segment_reduce`` and then added once: a fixed
    order, so the result is the same on every run (``index_add_`` on CUDA
    adds with atomics in arrival order). ``out`` may be a strided view."""
    if index.numel() == 0:
        return out
    idx = index.to(device=out.device, dtype=torch.int64).reshape(-1)
    width = int(source[0].numel())
    sidx, order = torch.sort(idx, stable=True)
    uniq, counts = torch.unique_consecutive(sidx, return_counts=True)
    ptr = torch.zeros(uniq.numel() + 1, dtype=torch.int32, device=out.device)
    ptr[1:] = torch.cumsum(counts, 0).to(torch.int32)
    src = (order * width).to(torch.int32)
    seg = L.Segments(uniq.numel(), width, 1, 0, ptr.data_ptr(), src.data_ptr())
    values = source.reshape(-1, width).to(device=out.device, dtype=torch.float64).contiguous()
    sums = torch.empty((uniq.numel(), width), dtype=torch.float64, device=out.device)
    segment_reduce(seg, values, sums)
    out[uniq] = out[uniq] + sums.view(-1, *out.shape[1:]).to(out.dtype)
    return out
